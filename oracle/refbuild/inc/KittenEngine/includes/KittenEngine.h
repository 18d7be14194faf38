// Replacement for KittenEngine/includes/KittenEngine.h used only by the recipe that compiles
// the reference's simulator sources for parity checks (test infrastructure).
//
// The real header pulls in the whole engine (OpenGL loader, windowing, asset and rendering
// modules).  The simulator (KittenEngine/YarnBall) needs only the math modules, which are
// included here unchanged from the reference, plus the names of three rendering types it holds
// pointers to.  Rendering stays off: the GL loader's function pointers, which the simulator
// tests before its rendering set-up (YarnBall.cu:172,191), are null as they are before any GL
// context exists, so those branches never run.  Nothing graphics-related is loaded.
#pragma once
#include <cfloat>
#include <cstddef>
#include <stdexcept>
#include <vector>

#include "KittenEngine/includes/modules/Common.h"
#include "KittenEngine/includes/modules/Bound.h"
#include "KittenEngine/includes/modules/Rotor.h"
#include "KittenEngine/includes/modules/SymMat.h"

namespace Kitten {
struct Mesh {};
struct ComputeBuffer {
    ComputeBuffer(size_t, size_t) {}
};
inline Mesh* genCylMesh(int, int, bool) { return nullptr; }
}  // namespace Kitten

namespace Kit = Kitten;

static const void* const glGetString = nullptr;
static const void* const glGetStringi = nullptr;
