// The binding that puts the B200 liquid step under the reference's own
// Scene<3> (Scene.cpp:13-20): the reference's "LiquidModel.h" is replaced by
// this header, and Scene<3> -- unchanged -- constructs, configures and owns
// the GPU model through the same calls it makes on its own LiquidModel<3>:
// LiquidModel<3>(const Scene<3>&), SetBoundary(BaseBoundary<3>*), Init,
// PreStep / Step / PostStep, GetCFL, GetParticleSystem, Render.
#pragma once

#include "Definition.h"
#include "Boundary.h"
#include "Scene.h"
#include "lhi_liquid.hpp"

template <int DIM>
class LiquidModel;

template <>
class LiquidModel<3> : public lhi_b200::LiquidModel<3> {
public:
    explicit LiquidModel(const Scene<3>& scene) : lhi_b200::LiquidModel<3>(scene) {}
};
