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
    chain_start();
    const int tid = threadIdx.x;
    if (tid == 0) {
        // read at once into registers, updated there, written back in one go
        swe_clock cl = *c;
        const uint32_t red_status = red[2], red_dt = red[3];
        s_record_row = -1;
        if (cl.active) {
            // The step that just ran (solver.py:627-632, :765-768).
            const uint32_t st = red_status;
            const float dt = __uint_as_float(red_dt);
            if (st & (SWE_S_NONFINITE_STATE | SWE_S_NONFINITE_DT | SWE_S_NONPOSITIVE_DT)) {
                cl.state = SWE_CLOCK_FAILED;
                cl.dt_status = st;
                cl.last_dt = dt;
                cl.active = 0;
            } else {
                double elapsed = cl.elapsed + (double)dt;
                if (elapsed > cl.duration && elapsed - cl.duration <= cl.tolerance) elapsed = cl.duration;
                cl.elapsed = elapsed;
                cl.last_dt = dt;
                cl.steps += 1;
                if (gauges && gauge_rows > 0) {
                    const int row = (cl.steps - 1) % gauge_rows;
                    gauges[(size_t)row * (2 + ngauge)] = cl.start + elapsed;
                    gauges[(size_t)row * (2 + ngauge) + 1] = (double)dt;
                    s_record_row = row;
                }
            }
        }
        if (cl.state == SWE_CLOCK_RUNNING) {
            // The next step (solver.py:741-760).
            // The loop runs out of iterations before it checks the remaining
            // time again, so max_steps is tested first.
            const double remaining = cl.duration - cl.elapsed;
            if (cl.steps >= cl.max_steps) {
                cl.state = SWE_CLOCK_MAXSTEPS;
                cl.active = 0;
            } else if (remaining <= cl.tolerance) {
                cl.state = SWE_CLOCK_DONE;
                cl.active = 0;
            } else {
                double step_max_dt = remaining;
                if (cl.max_dt_cap > 0.0 && cl.max_dt_cap < remaining) step_max_dt = cl.max_dt_cap;
                cl.max_dt = (float)step_max_dt;
                const double current = cl.start + cl.elapsed;
                if (nseries > 0) {
                    const float lev = interpolate_level(series_t, series_w, nseries, (float)current);
                    cl.level = lev;
                    level_out[0] = lev;
                }
                red[0] = 0u;
                red[1] = 0u;
                red[2] = 0u;
                cl.active = 1;
            }
        } else {
            cl.active = 0;
        }
        *c = cl;
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

// The gauge run's clock: each output interval is one forward() call of
// duration out_dt with its own level (run mode), or a re-run of recorded
// steps (replay mode).  Same double-precision bookkeeping as clock_kernel.
__global__ void run_clock_kernel(swe_run_clock* rc, uint32_t* red, const float* levels, int levelB,
                                 float* level_out, const float* U, const float* bed, int bedB,
                                 int B, int ny, int nx, const int32_t* gauge_cells, int ngauge,
                                 float* gauge_out, float* step_dt, int32_t* step_code) {
    __shared__ int s_record;  // interval whose gauges are read from U, or -1
    __shared__ int s_level;   // interval whose level the next step uses, or -1
    chain_start();
    const int tid = threadIdx.x;
    if (tid == 0) {
        // the clock and the step's status and dt are read at once into
        // registers, updated there and written back in one go (a chain of
        // dependent global accesses on one thread is the kernel's latency)
        swe_run_clock r = *rc;
        swe_clock& cl = r.base;
        const uint32_t red_status = red[2], red_dt = red[3];
        s_record = -1;
        s_level = -1;
        if (r.replay) {
            if (cl.active) cl.steps += 1;
            const int s = cl.steps;
            if (s < r.replay_end && s < r.record_cap) {
                cl.max_dt = step_dt[s];
                s_level = step_code[s] >> 1;
                red[0] = 0u;
                red[1] = 0u;
                red[2] = 0u;
                cl.active = 1;
            } else {
                cl.active = 0;
            }
        } else {
            if (cl.active) {
                const uint32_t st = red_status;
                const float dt = __uint_as_float(red_dt);
                if (st & (SWE_S_NONFINITE_STATE | SWE_S_NONFINITE_DT | SWE_S_NONPOSITIVE_DT)) {
                    cl.state = SWE_CLOCK_FAILED;
                    cl.dt_status = st;
                    cl.last_dt = dt;
                } else {
                    double elapsed = cl.elapsed + (double)dt;
                    if (elapsed > cl.duration && elapsed - cl.duration <= cl.tolerance)
                        elapsed = cl.duration;
                    cl.last_dt = dt;
                    const int s = cl.steps;
                    const bool ends = cl.duration - elapsed <= cl.tolerance;
                    if (s < r.record_cap) {
                        step_dt[s] = dt;
                        step_code[s] = 2 * r.chunk + (ends ? 1 : 0);
                    }
                    cl.steps = s + 1;
                    r.chunk_steps += 1;
                    cl.elapsed = elapsed;
                    if (ends) {
                        s_record = r.chunk;
                        r.chunk += 1;
                        r.chunk_steps = 0;
                        cl.elapsed = 0.0;
                    }
                }
            }
            if (cl.state == SWE_CLOCK_RUNNING) {
                if (r.chunk >= r.n_out) {
                    cl.state = SWE_CLOCK_DONE;
                } else if (cl.steps >= r.record_cap) {
                    cl.state = SWE_CLOCK_RECORD_FULL;
                } else if (r.chunk_steps >= cl.max_steps) {
                    cl.state = SWE_CLOCK_MAXSTEPS;
                } else {
                    // An interval that has not ended has remaining > tolerance.
                    const double remaining = cl.duration - cl.elapsed;
                    double step_max_dt = remaining;
                    if (cl.max_dt_cap > 0.0 && cl.max_dt_cap < remaining) step_max_dt = cl.max_dt_cap;
                    cl.max_dt = (float)step_max_dt;
                    s_level = r.chunk;
                    red[0] = 0u;
                    red[1] = 0u;
                    red[2] = 0u;
                }
            }
            cl.active = cl.state == SWE_CLOCK_RUNNING ? 1 : 0;
        }
        *rc = r;
    }
    __syncthreads();
    const int rec = s_record, lev = s_level;
    if (rec >= 0) {  // eta = h + bed at the gauges (after the interval's last step)
        const size_t plane = (size_t)ny * nx;
        for (int k = tid; k < B * ngauge; k += blockDim.x) {
            const int b = k / ngauge, g = k - b * ngauge;
            const size_t cell = (size_t)gauge_cells[2 * g] * nx + gauge_cells[2 * g + 1];
            const float z = bed[(bedB == 1 ? 0 : (size_t)b) * plane + cell];
            gauge_out[((size_t)b * rc->n_out + rec) * ngauge + g] = U[(size_t)b * 3 * plane + cell] + z;
        }
    }
    if (lev >= 0)
        for (int b = tid; b < levelB; b += blockDim.x) level_out[b] = levels[(size_t)lev * levelB + b];
}

// lam[b,0,cell_g] += g_gauge[b, c, g]; one thread per batch member, gauges in
// order, so repeated gauge cells accumulate deterministically.
__global__ void gauge_adjoint_kernel(float* lam, int B, int ny, int nx, const int32_t* gauge_cells,
                                     int ngauge, const float* g_gauge, int n_out, int c) {
    const size_t plane = (size_t)ny * nx;
    for (int b = threadIdx.x; b < B; b += blockDim.x)
        for (int g = 0; g < ngauge; ++g) {
            const size_t cell = (size_t)gauge_cells[2 * g] * nx + gauge_cells[2 * g + 1];
            lam[(size_t)b * 3 * plane + cell] += g_gauge[((size_t)b * n_out + c) * ngauge + g];
        }
}

__global__ void gauge_adjoint_prep_kernel(const int32_t* cursor, const float* step_dt,
                                          const int32_t* step_code, const float* levels, int levelB,
                                          float* dt_out, float* level_out, float* lam, int B, int ny,
                                          int nx, const int32_t* gauge_cells, int ngauge,
                                          const float* g_gauge, int n_out, int nsteps) {
    chain_start();
    const int s = *cursor;
    if (s < 0 || s >= nsteps) return;  // outside the record: nothing to set up
    const int code = step_code[s];
    const int c = code >> 1;
    if (threadIdx.x == 0) dt_out[0] = step_dt[s];
    for (int b = threadIdx.x; b < levelB; b += blockDim.x) level_out[b] = levels[(size_t)c * levelB + b];
    if (code & 1) {
        const size_t plane = (size_t)ny * nx;
        for (int b = threadIdx.x; b < B; b += blockDim.x)
            for (int g = 0; g < ngauge; ++g) {
                const size_t cell = (size_t)gauge_cells[2 * g] * nx + gauge_cells[2 * g + 1];
                lam[(size_t)b * 3 * plane + cell] += g_gauge[((size_t)b * n_out + c) * ngauge + g];
            }
    }
}

// One warp per batch member sums its partial sums in a fixed order.
__global__ void gauge_adjoint_post_kernel(int32_t* cursor, const int32_t* step_code,
                                          const float* parts, int nparts, int B, int blocks,
                                          int levelB, float* g_levels, int nsteps) {
    __shared__ float s_sum[32];
    __shared__ int s_step;
    chain_start();
    if (threadIdx.x == 0) s_step = *cursor;
    __syncthreads();  // every thread has the step before thread 0 moves the cursor
    const int s = s_step;
    if (s < 0 || s >= nsteps) return;
    const int c = step_code[s] >> 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    float total = 0.0f;  // levelB == 1: sum over members (thread 0)
    for (int b0 = 0; b0 < B; b0 += nw) {
        const int b = b0 + warp;
        float v = 0.0f;
        if (b < B)
            for (int q = 0; q < nparts; ++q)
                for (int k = lane; k < blocks; k += 32) v += parts[((size_t)q * B + b) * blocks + k];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (levelB > 1) {
            if (b < B && lane == 0) g_levels[(size_t)c * levelB + b] += v;
        } else {
            if (lane == 0) s_sum[warp] = b < B ? v : 0.0f;
            __syncthreads();
            if (threadIdx.x == 0)
                for (int w = 0; w < nw; ++w) total += s_sum[w];
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        if (levelB == 1) g_levels[c] += total;
        *cursor = s - 1;
    }
}

}  // namespace
}  // namespace swe

using namespace swe;

extern "C" int swe_gauge_adjoint_prep_f32(const int32_t* cursor, const float* step_dt,
                                          const int32_t* step_code, const float* levels, int levelB,
                                          float* dt_out, float* level_out, float* lam, int B, int ny,
                                          int nx, const int32_t* gauge_cells, int ngauge,
                                          const float* g_gauge, int n_out, int nsteps,
                                          void* stream) {
    if (!cursor || !step_dt || !step_code || !levels || levelB < 1 || !dt_out || !level_out || !lam ||
        B < 1 || ny < 1 || nx < 1 || ngauge < 0 || n_out < 1 || nsteps < 0)
        return SWE_EARG;
    if (ngauge > 0 && (!gauge_cells || !g_gauge)) return SWE_EARG;
    const cudaError_t e = launch_chained(gauge_adjoint_prep_kernel, dim3(1), dim3(128),
                                         (cudaStream_t)stream, cursor, step_dt, step_code, levels,
                                         levelB, dt_out, level_out, lam, B, ny, nx, gauge_cells, ngauge,
                                         g_gauge, n_out, nsteps);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int swe_gauge_adjoint_post_f32(int32_t* cursor, const int32_t* step_code,
                                          const float* parts, int nparts, int B, int blocks,
                                          int levelB, float* g_levels, int nsteps, void* stream) {
    if (!cursor || !step_code || !parts || nparts < 1 || B < 1 || blocks < 1 || !g_levels ||
        (levelB != 1 && levelB != B) || nsteps < 0)
        return SWE_EARG;
    const cudaError_t e = launch_chained(gauge_adjoint_post_kernel, dim3(1), dim3(256),
                                         (cudaStream_t)stream, cursor, step_code, parts, nparts, B,
                                         blocks, levelB, g_levels, nsteps);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int swe_run_clock_f32(swe_run_clock* clock, uint32_t* red, const float* levels,
                                 int levelB, float* level_out, const float* U, const float* bed,
                                 int bedB, int B, int ny, int nx, const int32_t* gauge_cells,
                                 int ngauge, float* gauge_out, float* step_dt, int32_t* step_code,
                                 void* stream) {
    if (!clock || !red || !levels || !level_out || levelB < 1 || !step_dt || !step_code)
        return SWE_EARG;
    if (B < 1 || ny < 1 || nx < 1 || ngauge < 0 || !U) return SWE_EARG;
    if (levelB != 1 && levelB != B) return SWE_EARG;
    if (ngauge > 0 && (!gauge_cells || !gauge_out || !bed || (bedB != 1 && bedB != B)))
        return SWE_EARG;
    const cudaError_t e = launch_chained(run_clock_kernel, dim3(1), dim3(128), (cudaStream_t)stream,
                                         clock, red, levels, levelB, level_out, U, bed, bedB, B, ny,
                                         nx, gauge_cells, ngauge, gauge_out, step_dt, step_code);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int swe_gauge_adjoint_f32(float* lam, int B, int ny, int nx, const int32_t* gauge_cells,
                                     int ngauge, const float* g_gauge, int n_out, int c,
                                     void* stream) {
    if (!lam || B < 1 || ny < 1 || nx < 1 || ngauge < 0 || n_out < 1 || c < 0 || c >= n_out)
        return SWE_EARG;
    if (ngauge == 0) return SWE_OK;
    if (!gauge_cells || !g_gauge) return SWE_EARG;
    gauge_adjoint_kernel<<<1, 128, 0, (cudaStream_t)stream>>>(lam, B, ny, nx, gauge_cells, ngauge,
                                                              g_gauge, n_out, c);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int swe_clock_f32(swe_clock* clock, uint32_t* red, const float* series_t,
                             const float* series_w, int nseries, float* level_out, const float* U,
                             int ny, int nx, const int32_t* gauge_cells, int ngauge, double* gauges,
                             int gauge_rows, void* stream) {
    if (!clock || !red || nseries < 0 || ngauge < 0) return SWE_EARG;
    if (nseries > 0 && (!series_t || !series_w || !level_out)) return SWE_EARG;
    if (ngauge > 0 && gauges && (!gauge_cells || !U || ny < 1 || nx < 1)) return SWE_EARG;
    const cudaError_t e = launch_chained(clock_kernel, dim3(1), dim3(128), (cudaStream_t)stream, clock,
                                         red, series_t, series_w, nseries, level_out, U, ny, nx,
                                         gauge_cells, ngauge, gauges, gauge_rows);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}
