/*
 * swe_oracle.h -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU restatement in plain C of DiffSWE2d's explicit finite-volume step, used
 * by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg to check
 * the CUDA path.  Nothing in diffswe2d_b200/ links or calls this library.
 *
 * Every function restates one reference function, evaluating the same
 * expression trees in the same order in the given precision (float or
 * double), with IEEE correctly-rounded +,-,*,/ and sqrt and no FMA
 * contraction.  Two reference operations are not correctly rounded on the
 * CPU build of PyTorch the reference runs on (AVX-512 sqrt and pow); the
 * oracle uses the correctly-rounded values instead, so it agrees with the
 * reference bit-for-bit except where one of those two operations differs
 * by an ulp.  tests/test_oracle.py measures that agreement against golden
 * outputs of the reference itself.
 *
 * Array layout: NCHW, row-major, contiguous.  U is [B,3,ny,nx]; bed and
 * roughness are [1 or B,1,ny,nx]; per-batch boundary values are arrays of B.
 */
#ifndef SWE_ORACLE_H
#define SWE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary codes, in the order of the reference's _VALID_BOUNDARY_TYPES
 * (src/boundary.py:11-18). */
enum {
    ORC_BC_TRANSMISSIVE = 0,
    ORC_BC_PERIODIC = 1,
    ORC_BC_CONSTANT = 2,
    ORC_BC_WATER_LEVEL = 3,
    ORC_BC_WALL = 4,
    ORC_BC_ABSORBING = 5,
};

/* Mirrors SWEConfig (src/config.py:4-28) plus the grid spacing. */
typedef struct {
    double gravity, dry_depth, epsilon, cfl, theta, dx, dy;
    double constant_value; /* value of "constant" boundaries */
    int32_t bc_left, bc_right, bc_top, bc_bottom;
    int32_t water_slope_reset, positivity_limiter, apply_friction;
    int32_t friction_model; /* 0 = manning, 1 = roughness length */
} orc_params;

#define ORC_DECLARE(R, SFX)                                                   \
    int orc_ghost_cells_##SFX(const R* U, const R* bed, int B, int bedB,     \
                              int ny, int nx, int ng, const orc_params* p,   \
                              const R* level, const R* cval, R* Up, R* zp);  \
    int orc_reconstruction_##SFX(const R* Up, const R* zp, int B, int zB,    \
                                 int H, int W, int dim, const orc_params* p, \
                                 R* UL, R* UR, R* sL, R* sR);                \
    int orc_hll_flux_##SFX(const R* UL, const R* UR, int B, int H, int W,    \
                           int normal_y, const orc_params* p, R* flux,       \
                           R* speed);                                        \
    int orc_primitive_##SFX(const R* U, int B, int H, int W,                 \
                            const orc_params* p, R* h, R* u, R* v, R* c);    \
    int orc_limited_increment_##SFX(const R* q, int B, int C, int H, int W,  \
                                    int dim, double theta, R* out);          \
    int orc_spatial_operator_##SFX(const R* U, const R* bed, int B,          \
                                   int bedB, int ny, int nx,                 \
                                   const orc_params* p, const R* level,      \
                                   const R* rain, const R* infil, R* rhs,    \
                                   R* ax, R* ay);                            \
    int orc_clean_and_limit_##SFX(const R* old, const R* cand, int B,        \
                                  int ny, int nx, const orc_params* p,       \
                                  R* out);                                   \
    int orc_manning_##SFX(const R* U, const R* n, int B, int nB, int ny,     \
                          int nx, R dt, double dry_depth, double epsilon,    \
                          R* out);                                           \
    int orc_roughness_friction_##SFX(const R* U, const R* z0, int B, int nB, \
                                     int ny, int nx, R dt, double dry_depth, \
                                     double epsilon, R* out);                \
    int orc_step_##SFX(const R* U, const R* bed, int bedB, const R* n,       \
                       int nB, int B, int ny, int nx, const orc_params* p,   \
                       const R* level, R max_dt, const R* infil, R* U_out,   \
                       R* dt_out);                                           \
    int orc_step_forced_##SFX(const R* U, const R* bed, int bedB,            \
                              const R* n, int nB, int B, int ny, int nx,     \
                              const orc_params* p, const R* level, R max_dt, \
                              const R* rain0, const R* rain1,                \
                              const R* infil, R* U_out, R* dt_out);

ORC_DECLARE(float, f32)
ORC_DECLARE(double, f64)

int orc_num_threads(void);

#ifdef __cplusplus
}
#endif

#endif /* SWE_ORACLE_H */
