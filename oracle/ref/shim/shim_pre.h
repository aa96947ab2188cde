// Test-infrastructure shim, force-included (-include) into every reference
// translation unit compiled by oracle/ref/Makefile.
//
// The reference's GUI header (src/gui.cuh) pulls in ImGui, GLFW, glad, glm and
// CUDA-GL interop, none of which exist on this machine or the GPU box. The SPH
// hot path only touches three GUI members (particles.cu:5-90, buffer.cuh:60);
// this stub provides them and throws if they are ever called, so the headless
// oracle build can never take an interop path by accident.
#pragma once
#define GUI_H_
#define __CUDA_GL_INTEROP_H__
#include <cfloat>
#include <cstdint>
#include <stdexcept>
#include <sys/types.h>

class Particles;
class GUI {
public:
    uint N { 1 };
    void initialize_buffers(Particles&)
    {
        throw std::runtime_error("GUI is not available in the oracle build");
    }
    void resize_mapped_buffers(uint, Particles&)
    {
        throw std::runtime_error("GUI is not available in the oracle build");
    }
    float* resize_pos_component(uint, Particles&, int)
    {
        throw std::runtime_error("GUI is not available in the oracle build");
    }
};

// src/scene/sample_boundary.cuh:82 names BoundarySamples before
// src/scene/scene.cuh:29 defines it (the reference relies on includer order).
struct BoundarySamples;
