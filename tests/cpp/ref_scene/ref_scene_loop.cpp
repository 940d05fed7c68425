// The reference's frame loop (main.cpp:14-55, without the window and the
// render) over the reference's own Scene<3> (Scene.cpp, compiled unchanged
// from the reference tree) whose LiquidModel<3> is the B200 liquid step
// (binding/LiquidModel.h).
//
//   ref_scene_loop <config.json> <steps> <positions.bin>
//
// Init(), then <steps> x (PreStep, Step, PostStep, dt = GetCFL()) from
// dt = 0.01 as main.cpp does; writes the particle positions (float xyz) and
// prints one JSON line.
#include <cstdio>
#include <string>
#include <vector>

#include "Definition.h"
#include "Scene.h"
#include "LiquidModel.h"

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s config.json steps positions.bin\n", argv[0]);
        return 1;
    }
    try {
        Scene<3> scene(argv[1]);
        LiquidModel<3>& liquidModel = scene.GetLiquidModel();
        liquidModel.Init();
        const long long spawned = liquidModel.GetParticleSystem().NumParticles();
        Scalar dt = 0.01;
        std::vector<double> dts;
        const int steps = std::stoi(argv[2]);
        for (int s = 0; s < steps; ++s) {
            dts.push_back(dt);
            liquidModel.PreStep(dt);
            liquidModel.Step(dt);
            liquidModel.PostStep(dt);
            dt = liquidModel.GetCFL();
        }
        const std::vector<Scalar> pos = liquidModel.GetParticleSystem().GetPositions();
        FILE* f = std::fopen(argv[3], "wb");
        if (!f || std::fwrite(pos.data(), sizeof(Scalar), pos.size(), f) != pos.size()) {
            std::fprintf(stderr, "cannot write %s\n", argv[3]);
            return 1;
        }
        std::fclose(f);
        std::printf("{\"particles\": %lld, \"spawned\": %lld, \"steps\": %d, \"dt\": [", (long long)(pos.size() / 3),
                    spawned, steps);
        for (size_t i = 0; i < dts.size(); ++i) std::printf("%s%.9g", i ? ", " : "", dts[i]);
        std::printf("]}\n");
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 2;
    }
    return 0;
}
