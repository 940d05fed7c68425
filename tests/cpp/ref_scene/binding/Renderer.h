// Headless stand-in for the reference's Renderer.h in this test build only:
// no display or OpenGL is available, and the liquid step does not render.
// Scene<3>::PlaySimulation (Scene.cpp:24-45) is the only user in Scene.cpp.
#pragma once

class Renderer {
public:
    static Renderer& GetInstance() {
        static Renderer r;
        return r;
    }
    void ClearScreen() const {}
    void LoadScreen() const {}
};
