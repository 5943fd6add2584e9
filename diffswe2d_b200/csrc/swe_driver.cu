// swe_driver.cu -- the time-loop bookkeeping of SWE2D.forward on the device.
//
// The reference's forward() (src/solver.py:680-779) is a Python loop that
// synchronises with the GPU several times per step.  Here the loop state is
// a swe_clock in device memory and one single-block kernel advances it
// between steps, so a host can enqueue (or capture in a CUDA graph) many
// steps and read the clock once per chunk.  The arithmetic is the
// reference's: double-precision elapsed/remaining time, float32 max_dt and
// float32 interpolation of the boundary series.
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "swe_common.cuh"

namespace swe {
namespace {

// SWE2D._interpolate_dynamic_boundary (src/solver.py:391-415) in float32:
// index = searchsorted(times, t, right=False) clamped to [1, n-1].
__device__ float interpolate_level(const float* times, const float* levels, int n, float t) {
    if (n == 1) return levels[0];
    int lo = 0, hi = n;
    while (lo < hi) {  // first index with times[i] >= t
        const int mid = (lo + hi) >> 1;
        if (times[mid] < t) lo = mid + 1;
        else hi = mid;
    }
    const int idx = min(max(lo, 1), n - 1);
    const float t0 = times[idx - 1], t1 = times[idx];
    const float w0 = levels[idx - 1], w1 = levels[idx];
    const float span = t1 - t0;
    const float weight = __fdiv_rn(t - t0, fmaxf(span, FLT_EPSILON));
    return w0 + weight * (w1 - w0);
}

__global__ void clock_kernel(swe_clock* c, uint32_t* red, const float* series_t,
                             const float* series_w, int nseries, float* level_out, const float* U,
                             int ny, int nx, const int32_t* gauge_cells, int ngauge, double* gauges,
                             int gauge_rows) {
    __shared__ int s_record_row;
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_record_row = -1;
        if (c->active) {
            // The step that just ran (solver.py:627-632, :765-768).
            const uint32_t st = red[2];
            const float dt = __uint_as_float(red[3]);
            if (st & (SWE_S_NONFINITE_STATE | SWE_S_NONFINITE_DT | SWE_S_NONPOSITIVE_DT)) {
                c->state = SWE_CLOCK_FAILED;
                c->dt_status = st;
                c->last_dt = dt;
                c->active = 0;
            } else {
                double elapsed = c->elapsed + (double)dt;
                if (elapsed > c->duration && elapsed - c->duration <= c->tolerance) elapsed = c->duration;
                c->elapsed = elapsed;
                c->last_dt = dt;
                c->steps += 1;
                if (gauges && gauge_rows > 0) {
                    const int row = (c->steps - 1) % gauge_rows;
                    gauges[(size_t)row * (2 + ngauge)] = c->start + elapsed;
                    gauges[(size_t)row * (2 + ngauge) + 1] = (double)dt;
                    s_record_row = row;
                }
            }
        }
        if (c->state == SWE_CLOCK_RUNNING) {
            // The next step (solver.py:741-760).
            // The loop runs out of iterations before it checks the remaining
            // time again, so max_steps is tested first.
            const double remaining = c->duration - c->elapsed;
            if (c->steps >= c->max_steps) {
                c->state = SWE_CLOCK_MAXSTEPS;
                c->active = 0;
            } else if (remaining <= c->tolerance) {
                c->state = SWE_CLOCK_DONE;
                c->active = 0;
            } else {
                double step_max_dt = remaining;
                if (c->max_dt_cap > 0.0 && c->max_dt_cap < remaining) step_max_dt = c->max_dt_cap;
                c->max_dt = (float)step_max_dt;
                const double current = c->start + c->elapsed;
                if (nseries > 0) {
                    const float lev = interpolate_level(series_t, series_w, nseries, (float)current);
                    c->level = lev;
                    level_out[0] = lev;
                }
                red[0] = 0u;
                red[1] = 0u;
                red[2] = 0u;
                c->active = 1;
            }
        } else {
            c->active = 0;
        }
    }
    __syncthreads();
    const int row = s_record_row;
    if (row >= 0) {  // depth of batch 0 at each gauge cell (solver.py:798)
        for (int g = tid; g < ngauge; g += blockDim.x) {
            const int iy = gauge_cells[2 * g], ix = gauge_cells[2 * g + 1];
            gauges[(size_t)row * (2 + ngauge) + 2 + g] = (double)U[(size_t)iy * nx + ix];
        }
    }
}

}  // namespace
}  // namespace swe

using namespace swe;

extern "C" int swe_clock_f32(swe_clock* clock, uint32_t* red, const float* series_t,
                             const float* series_w, int nseries, float* level_out, const float* U,
                             int ny, int nx, const int32_t* gauge_cells, int ngauge, double* gauges,
                             int gauge_rows, void* stream) {
    if (!clock || !red || nseries < 0 || ngauge < 0) return SWE_EARG;
    if (nseries > 0 && (!series_t || !series_w || !level_out)) return SWE_EARG;
    if (ngauge > 0 && gauges && (!gauge_cells || !U || ny < 1 || nx < 1)) return SWE_EARG;
    clock_kernel<<<1, 128, 0, (cudaStream_t)stream>>>(clock, red, series_t, series_w, nseries, level_out,
                                                      U, ny, nx, gauge_cells, ngauge, gauges,
                                                      gauge_rows);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}
