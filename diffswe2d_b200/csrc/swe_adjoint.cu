// swe_adjoint.cu -- adjoint (vector-Jacobian product) of one SWE2D.step on
// sm_100a, matching the reference's autograd gradient (src/solver.py:572-663
// under PyTorch autograd; dt detached, solver.py:626).
//
// The step is S(U) -> k1, P = C(U, U + dt/2 k1), S(P) -> k2,
// Q = C(U, U + dt k2), U' = F(Q, n).  Its adjoint runs, per step:
//   swe_adj_pointwise_f32(mode 0, or 3 writing lamU): friction and corrector clean-up adjoints
//       (friction.py:12-131, solver.py:547-570) -> lamU, lam_k2, lam_n
//   swe_adj_stage2_f32 at P:       adjoint of the spatial operator and of
//       the predictor clean-up (solver.py:639) -> lamU, lam_k1
//   swe_adj_spatial_f32 on U:      -> lamU
// (swe_adj_stage2_f32 is swe_adj_spatial_f32 into a zeroed lam_P followed
// by swe_adj_pointwise_f32 mode 1, in two launches instead of three.)
// The kernels are in swe_adjoint_kernels.cuh.  This file holds the C ABI and
// the IEEE instantiation (ExactMath, for SWE_ARITH_EXACT parameters);
// parameters with SWE_ARITH_FAST run the FastMath instantiation of
// swe_adjoint_fast.cu.
#include "swe_adjoint_kernels.cuh"

using namespace swe;

namespace {

// The spatial adjoint's arguments (checked), without the fused-predictor part.
int adj_args(AdjArgs& a, const float* S, const float* bed, int bedB, int B, int ny, int nx,
             const swe_params* p, const float* level, int levelB, const float* lam_rhs,
             float* scratch_cx, float* scratch_cy, float* level_part, int level_blocks,
             float* lam_bed) {
    if (!S || !bed || !level || !lam_rhs || !scratch_cx || !scratch_cy || !level_part)
        return SWE_EARG;
    if (!valid_params(p) || B < 1 || ny < 2 || nx < 2 || level_blocks < 1) return SWE_EARG;
    if ((bedB != 1 && bedB != B) || (levelB != 1 && levelB != B) || B > 65535) return SWE_EARG;
    a = AdjArgs{};
    a.S = S;
    a.bed = bed;
    a.level = level;
    a.lrhs = lam_rhs;
    a.cx = scratch_cx;
    a.cy = scratch_cy;
    a.llevel_part = level_part;
    a.lbed = lam_bed;
    a.B = B;
    a.bedB = bedB;
    a.levelB = levelB;
    a.ny = ny;
    a.nx = nx;
    a.bc[0] = p->bc_left;
    a.bc[1] = p->bc_right;
    a.bc[2] = p->bc_top;
    a.bc[3] = p->bc_bottom;
    a.cval = (float)p->constant_value;
    a.wsr = p->water_slope_reset;
    a.kc = make_consts(*p);
    a.positivity = p->positivity_limiter;
    return SWE_OK;
}

int run_spatial(const AdjArgs& a, const swe_params* p, int level_blocks, bool pred, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (p->arithmetic == SWE_ARITH_FAST) return fast_launch_adj_spatial(a, level_blocks, pred, s);
    return launch_adj_spatial<ExactMath>(a, level_blocks, pred, s);
}

int adj_spatial(const float* S, const float* bed, int bedB, int B, int ny, int nx,
                const swe_params* p, const float* level, int levelB, const float* lam_rhs,
                float* scratch_cx, float* scratch_cy, float* lam_S, float* level_part,
                int level_blocks, float* lam_bed, void* stream) {
    AdjArgs a;
    const int rc = adj_args(a, S, bed, bedB, B, ny, nx, p, level, levelB, lam_rhs, scratch_cx,
                            scratch_cy, level_part, level_blocks, lam_bed);
    if (rc != SWE_OK) return rc;
    if (!lam_S) return SWE_EARG;
    a.lS = lam_S;
    return run_spatial(a, p, level_blocks, false, stream);
}
}  // namespace

extern "C" int swe_adj_spatial_f32(const float* S, const float* bed, int bedB, int B, int ny, int nx,
                                   const swe_params* p, const float* level, int levelB,
                                   const float* lam_rhs, float* scratch_cx, float* scratch_cy,
                                   float* lam_S, float* level_part, int level_blocks,
                                   void* stream) {
    return adj_spatial(S, bed, bedB, B, ny, nx, p, level, levelB, lam_rhs, scratch_cx, scratch_cy,
                       lam_S, level_part, level_blocks, nullptr, stream);
}

extern "C" int swe_adj_spatial_bed_f32(const float* S, const float* bed, int bedB, int B, int ny,
                                       int nx, const swe_params* p, const float* level, int levelB,
                                       const float* lam_rhs, float* scratch_cx, float* scratch_cy,
                                       float* lam_S, float* level_part, int level_blocks,
                                       float* lam_bed, void* stream) {
    if (!lam_bed) return SWE_EARG;
    return adj_spatial(S, bed, bedB, B, ny, nx, p, level, levelB, lam_rhs, scratch_cx, scratch_cy,
                       lam_S, level_part, level_blocks, lam_bed, stream);
}

extern "C" int swe_adj_stage2_f32(const float* P, const float* U, const float* k1, const float* bed,
                                  int bedB, int B, int ny, int nx, const swe_params* p,
                                  const float* level, int levelB, const float* lam_k2,
                                  float* scratch_cx, float* scratch_cy, float dt,
                                  const float* dt_dev, float* lam_U, float* lam_k1,
                                  float* level_part, int level_blocks, float* lam_bed,
                                  void* stream) {
    AdjArgs a;
    const int rc = adj_args(a, P, bed, bedB, B, ny, nx, p, level, levelB, lam_k2, scratch_cx,
                            scratch_cy, level_part, level_blocks, lam_bed);
    if (rc != SWE_OK) return rc;
    if (!U || !k1 || !lam_U || !lam_k1) return SWE_EARG;
    a.U = U;
    a.k1 = k1;
    a.dt = dt;
    a.dt_dev = dt_dev;
    a.lU = lam_U;
    a.lk1 = lam_k1;
    return run_spatial(a, p, level_blocks, true, stream);
}

namespace {
int adj_pointwise(int mode, const float* U, const float* k, const float* n, int nB, int B, int ny,
                  int nx, const swe_params* p, float dt, const float* dt_dev, const float* lam_out,
                  float* lam_U, float* lam_k, float* lam_n, float* P_out, void* stream) {
    if (mode < 0 || mode > 3 || !U || !k || !valid_params(p) || B < 1 || ny < 1 || nx < 1)
        return SWE_EARG;
    if (mode == 2 && !P_out) return SWE_EARG;
    if (mode != 2 && (!lam_out || !lam_U || !lam_k)) return SWE_EARG;
    if ((mode == 0 || mode == 3) && p->apply_friction && (!n || !lam_n || (nB != 1 && nB != B)))
        return SWE_EARG;
    PwArgs a{};
    a.U = U;
    a.k = k;
    a.n = n;
    a.lout = lam_out;
    a.lU = lam_U;
    a.lk = lam_k;
    a.ln = lam_n;
    a.P = P_out;
    a.dt = dt;
    a.scale = (mode == 0 || mode == 3) ? dt : 0.5f * dt;
    a.dt_dev = dt_dev;
    a.B = B;
    a.nB = nB;
    a.ny = ny;
    a.nx = nx;
    a.mode = mode;
    a.positivity = p->positivity_limiter;
    a.friction = p->apply_friction;
    a.friction_model = p->friction_model;
    a.kc = make_consts(*p);
    cudaStream_t s = (cudaStream_t)stream;
    if (p->arithmetic == SWE_ARITH_FAST) return fast_launch_adj_pointwise(a, s);
    return launch_adj_pointwise<ExactMath>(a, s);
}
}  // namespace

extern "C" int swe_adj_pointwise_f32(int mode, const float* U, const float* k, const float* n,
                                     int nB, int B, int ny, int nx, const swe_params* p, float dt,
                                     const float* lam_out, float* lam_U, float* lam_k,
                                     float* lam_n, float* P_out, void* stream) {
    return adj_pointwise(mode, U, k, n, nB, B, ny, nx, p, dt, nullptr, lam_out, lam_U, lam_k, lam_n,
                         P_out, stream);
}

extern "C" int swe_adj_pointwise_dev_f32(int mode, const float* U, const float* k, const float* n,
                                         int nB, int B, int ny, int nx, const swe_params* p,
                                         const float* dt_dev, const float* lam_out, float* lam_U,
                                         float* lam_k, float* lam_n, float* P_out, void* stream) {
    if (!dt_dev) return SWE_EARG;
    return adj_pointwise(mode, U, k, n, nB, B, ny, nx, p, 0.0f, dt_dev, lam_out, lam_U, lam_k, lam_n,
                         P_out, stream);
}
