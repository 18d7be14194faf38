// io.cuh - launchers for layout conversion, diagnostics and BVH root boxes (k_io.cu).
#pragma once
#include "engine.cuh"

namespace yb {
template <typename R>
void launch_convert_in(const Dev<R>& d, const void* hv, const float* hvel, const float* hq, const float* hqr,
                       const int* sceneOf, cudaStream_t s);
// Converts vertices [first, first+count) to the host layout (written at the same offsets).
template <typename R>
void launch_convert_out(const Dev<R>& d, void* hv, float* hvel, float* hq, int first, int count, cudaStream_t s);
template <typename R> void launch_relayout(const Dev<R>& d, const int* sceneOf, const int* delta, cudaStream_t s);
template <typename R> void launch_zero_vel(const Dev<R>& d, cudaStream_t s);
template <typename R>
void launch_state_f64(const Dev<R>& d, int buf, double* pos, double* vel, double* q, double* dx, cudaStream_t s);
template <typename R> void launch_scene_root_box(const Dev<R>& d, float* out, cudaStream_t s);
// Writes 8 doubles per block into part; returns the number of blocks.
template <typename R> int launch_diag(const Dev<R>& d, double* part, cudaStream_t s);
// Largest change of the Newton iterate made by the last iteration (which read buffer src and
// wrote src ^ 1), max over vertices of |dx_new - dx_old| in FP64, folded into *slot (the bit
// pattern of a non-negative double; zero it first).
template <typename R> void launch_iter_delta(const Dev<R>& d, int src, unsigned long long* slot, cudaStream_t s);
}  // namespace yb
