// No-op GLFW surface for compiling the reference headlessly.
// TEST INFRASTRUCTURE (reference cross-check build only).
#pragma once
struct GLFWwindow;
typedef void (*GLFWmousebuttonfun)(GLFWwindow*, int, int, int);
typedef void (*GLFWkeyfun)(GLFWwindow*, int, int, int, int);
inline GLFWmousebuttonfun glfwSetMouseButtonCallback(GLFWwindow*, GLFWmousebuttonfun f) { return f; }
inline GLFWkeyfun glfwSetKeyCallback(GLFWwindow*, GLFWkeyfun f) { return f; }
