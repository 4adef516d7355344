/*
 * kmhd_sph.h -- C-ABI of the B200 spherical-transform cycle.
 *
 * Drop-in boundary for Calypso's transform entry points.  Every entry point
 * takes plain pointers and sizes, returns an int status (KMHD_OK = 0) and never
 * exits; kmhd_strerror() turns a status into text.  The reference aborts via
 * calypso_MPI_abort instead (SOLVER_src/send_recv/calypso_mpi.f90:114).
 *
 * Spectral arrays use the reference's rj layout: d_rj(inod, icomp),
 * column-major, inod = j + J*k (j fastest, k = radius), leading dimension ld.
 * A vector field occupies three consecutive columns (S, dS/dr, T); the caller
 * names the first column of each field (cols_*), as ipol%i_velo etc. do in
 * MHD_src/sph_MHD/set_address_sph_trans_MHD.f90.  The j order is the
 * reference's single-domain order (m = -L..L, then l = |m|..L) unless
 * kmhd_sph_desc.idx_rj_lm gives (l, m) per j.
 * Grid arrays use the reference's rtp layout: fld_rtp(nnod_rtp, ncomp),
 * column-major, node = r + Nr*(theta + Ntheta*phi); a vector's three
 * columns are (r, theta, phi) components.
 * Paths are relative to MHD/Fortran_src/ of the reference.
 */
#ifndef KMHD_SPH_H
#define KMHD_SPH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum kmhd_status {
  KMHD_OK = 0,
  KMHD_ERR_ARG = 1,        /* invalid descriptor or argument */
  KMHD_ERR_SIZE = 2,       /* unsupported size (L, grid, field counts) */
  KMHD_ERR_CUDA = 3,       /* CUDA runtime error */
  KMHD_ERR_NOMEM = 4,      /* device allocation failed */
  KMHD_ERR_DEVICE = 5,     /* no sm_100 device */
  KMHD_ERR_TIMEOUT = 6,    /* bounded device wait expired (work queue) */
  KMHD_ERR_STATE = 7       /* call order / handle state */
};

enum kmhd_tier {
  KMHD_TIER_FP64 = 0,      /* FP64 Legendre GEMMs (DMMA), bit-faithful method   */
  KMHD_TIER_SPLIT_I8 = 1,  /* INT8-slice split products on tcgen05, <=1e-12     */
  KMHD_TIER_FP32ACC = 2    /* 4-slice INT8 split, 10 products on tcgen05, <=1e-6 */
};

enum kmhd_product_kind {
  KMHD_PROD_CROSS = 0,       /* fwd vector = coef * (bwd_vec[a] x bwd_vec[b])   */
  KMHD_PROD_VEC_SCALAR = 1,  /* fwd vector = coef * bwd_vec[a] * bwd_scl[b]     */
  KMHD_PROD_DOT = 2,         /* fwd scalar = coef * (bwd_vec[a] . bwd_vec[b])   */
  KMHD_PROD_SCALAR = 3       /* fwd scalar = coef * bwd_scl[a] * bwd_scl[b]     */
};

/* One grid-space product of the cycle; forward vectors are produced in list
 * order, then forward scalars.  Mirrors cal_cross_prod_w_coef_smp /
 * cal_vec_scalar_prod_w_coef_smp / cal_dot_prod_w_coef_smp
 * (CORE_src/BASE/cal_products_smp.f90) as called by nonlinear_terms_in_rtp
 * (MHD_src/sph_MHD/cal_nonlinear_sph_MHD.f90:64-128). */
typedef struct kmhd_product {
  int32_t kind;
  int32_t a, b;
  double coef;
} kmhd_product;

typedef struct kmhd_sph_desc {
  int32_t ltr;          /* truncation L (l_truncation)                         */
  int32_t nth;          /* Gauss-Legendre latitudes  (nidx_rtm(2))             */
  int32_t nph;          /* longitudes (nidx_rtp(3)), 2^a 3^b 5^c, > 2L         */
  int32_t nr;           /* radial points (nidx_rj(1))                          */
  const double *radius; /* [nr] host, radius_1d_rj_r                           */
  const int32_t *idx_rj_lm; /* [2*(L+1)^2] host (l, m) per rj j, or NULL       */
  int32_t nvector_b, nscalar_b;   /* rj -> rtp fields  (nvector_rj_2_rtp ...), <= 5 / 2 */
  int32_t nvector_f, nscalar_f;   /* rtp -> rj fields  (nvector_rtp_2_rj ...), <= 5 / 2 */
                                  /* split tiers: at most 6 fields per direction   */
  int32_t nproduct;               /* grid products for kmhd_sph_cycle          */
  const kmhd_product *products;   /* [nproduct] host                           */
  int32_t tier;                   /* enum kmhd_tier                            */
  int32_t nslice;                 /* split tiers: slices per operand, 0=default */
  int32_t device;                 /* CUDA device ordinal                       */
  int32_t flags;                  /* KMHD_FLAG_* bits, 0 = none                */
} kmhd_sph_desc;

typedef struct kmhd_sph kmhd_sph;

/* kmhd_sph_desc.flags: for the split tiers, on the first kmhd_sph_batch_cycle
 * call run three candidates on the call's own data -- the FP64 DMMA path, the
 * split path with the tier's full slice-product count (26 split, 10 fp32acc)
 * and the split path with the highest digit-pair group dropped (21, 6) --
 * compare the split outputs with the FP64 path's (max-norm relative error per
 * output column) and keep the fastest candidate whose error is at most a
 * quarter of the tier's bound (1e-12, 1e-6).  kmhd_sph_get_tuning reports the
 * choice, the times and the errors.  The reference times its Legendre variants
 * at start-up (select_legendre_transform,
 * MHD_src/sph_MHD/init_sphrical_transform_MHD.f90:201-345), without an error
 * check. */
#define KMHD_FLAG_AUTOTUNE 1
/* kmhd_sph_desc.flags, FP64 tier only: no stored P / dP tables; the Legendre
 * kernels generate P_l^m and dP_l^m/dtheta by the fixed-order recurrence as
 * they go, from O(L^2) coefficients, O(L Ntheta) start values and seeds every
 * 32 degrees (about 20x less memory than the O(L^2 Ntheta) tables).  Values
 * differ from the stored tables in the last bits only.  The reference stores
 * the tables (schmidt_poly_on_rtm_grid.f90:145-197). */
#define KMHD_FLAG_P_ON_THE_FLY 2

/* Pointer-location flag for data arguments. */
#define KMHD_PTR_DEVICE 0
#define KMHD_PTR_HOST 1

/* Builds the handle: Gauss nodes/weights, Schmidt P_l^m and dP_l^m/dtheta
 * tables (FP64 recurrence on the device), index tables and work buffers.
 * Replaces initialize_legendre_trans / init_legendre_rtm / set_sym_legendre_stack
 * / init_legendre_sym_matmul (PARALLEL_src/SPH_SHELL_src/init_sph_trans.f90:79-168,
 * t_legendre_work_sym_matmul.f90:150-262). */
int kmhd_sph_create(const kmhd_sph_desc *desc, kmhd_sph **handle);

/* Releases every device resource of the handle. */
int kmhd_sph_destroy(kmhd_sph *handle);

/* Binds a caller stream (cudaStream_t) for all subsequent calls; NULL = the
 * handle's own stream. */
int kmhd_sph_set_stream(kmhd_sph *handle, void *stream);

/* Backward transform: spectral fields -> grid.  Replaces sph_b_trans_w_coriolis
 * without Coriolis (MHD_src/sph_MHD/sph_trans_w_coriols.f90:113-187) and
 * sph_backward_transforms (PARALLEL_src/SPH_SHELL_src/t_sph_transforms.f90:74-123).
 * d_rj: ld >= J*nr; cols_b[nvector_b + nscalar_b] first column per field.
 * fld_rtp: nnod_rtp x (3*nvector_b + nscalar_b), column-major. */
int kmhd_sph_b_trans(kmhd_sph *handle, const double *d_rj, int64_t ld_rj,
                     const int32_t *cols_b, double *fld_rtp, int32_t ptr_kind);

/* Forward transform: grid forces -> spectral.  Replaces sph_f_trans_w_coriolis
 * without Coriolis (sph_trans_w_coriols.f90:189-246) and sph_forward_transforms
 * (t_sph_transforms.f90:250-297).  frc_rtp: nnod_rtp x (3*nvector_f + nscalar_f). */
int kmhd_sph_f_trans(kmhd_sph *handle, const double *frc_rtp, double *d_rj,
                     int64_t ld_rj, const int32_t *cols_f, int32_t ptr_kind);

/* Full cycle: backward transform, grid products, forward transform.  Replaces
 * the copy_mhd_spectr_to_send -> sph_b_trans -> nonlinear_terms_in_rtp ->
 * sph_f_trans -> copy_mhd_spectr_from_recv segment of nonlinear_by_pseudo_sph
 * (MHD_src/sph_MHD/cal_nonlinear.f90:118-171).  With host pointers and more
 * than 64 MiB of copies the call runs over radial chunks whose copies in and
 * out overlap the kernels (page-locked host memory overlaps; pageable memory
 * gives the same result more slowly); the result equals the device-pointer
 * call's, input and output columns may share one array, and only the whole
 * call is timed (kmhd_sph_last_timing stages 0..2 read 0). */
int kmhd_sph_cycle(kmhd_sph *handle, const double *d_rj_in, int64_t ld_in,
                   const int32_t *cols_b, double *d_rj_out, int64_t ld_out,
                   const int32_t *cols_f, int32_t ptr_kind);

/* Batched uneven instances: n cycles (device pointers) of possibly different
 * L, Nr and field counts.  Every instance runs on its own handle's stream; one
 * CUDA graph, captured on the first call and replayed while handles, pointers
 * and leading dimensions stay the same, forks them all and joins them, so small
 * instances fill the GPU together.  Handles created with KMHD_FLAG_AUTOTUNE
 * pick their Legendre path by timing on the first call.  Returns after all
 * instances finished.  Replaces n calls of the cycle; the reference has no
 * batched form. */
int kmhd_sph_batch_cycle(kmhd_sph **handles, int32_t n, const double *const *d_rj_in,
                         const int64_t *ld_in, const int32_t *const *cols_b,
                         double *const *d_rj_out, const int64_t *ld_out,
                         const int32_t *const *cols_f);

/* Stage times of the last call in ms (CUDA events): [0] Legendre bwd (label 22),
 * [1] FFT + products + FFT (labels 24 + nonlinear), [2] Legendre fwd (label 23),
 * [3] whole call.  Labels as in MHD_src/IO/init_sph_MHD_elapsed_label.f90:38-84. */
int kmhd_sph_last_timing(kmhd_sph *handle, double *ms4);

/* Per-launch times in ms (CUDA events on the handle's stream) of the last
 * kmhd_sph_cycle: [0] backward pack (FP64) or slicer (split tiers), [1]
 * backward Legendre GEMM, [2] FFT + products + FFT, [3] forward slicer (0 for
 * FP64), [4] forward Legendre GEMM.  KMHD_ERR_STATE if the last call was not
 * a cycle.  Finer-grained than the reference's elapsed labels
 * (MHD_src/IO/init_sph_MHD_elapsed_label.f90:38-84). */
int kmhd_sph_last_kernel_timing(kmhd_sph *handle, double *ms5);

/* Copies the device Gauss colatitudes/weights [nth] and the hemisphere
 * P / dP tables of order m ([nth_hemi x (L-m+1)], rows theta, cols l) to host
 * arrays, for parity checks of the set-up stage (with KMHD_FLAG_P_ON_THE_FLY:
 * the values the kernels generate). */
int kmhd_sph_get_tables(kmhd_sph *handle, int32_t m, double *colat, double *weight,
                        double *P, double *dP);

/* The FP64 cycle of kmhd_sph_cycle for callers that cannot allocate device
 * memory: a solver whose host framework owns the whole device pool, or a
 * time-step loop that must not call cudaMalloc/cudaFree (which can stall the
 * device) once set-up is over.  No handle is built: every work buffer --
 * Gauss/Schmidt tables, index maps, FFT twiddles, packed spectra and the
 * (m, theta, r) records -- lives in one static 32 MiB device array that the
 * library holds on every device it is loaded on until the process exits; the
 * tables are recomputed on each call.  desc->tier must be KMHD_TIER_FP64;
 * d_rj_in / d_rj_out are device pointers (cols_b / cols_f and desc's arrays
 * stay on the host); stream is a cudaStream_t (NULL = default stream) and the
 * call returns after it has been synchronised.  Returns KMHD_ERR_SIZE when the
 * problem needs more than the 32 MiB (about L = 31, Ntheta = 48, Nphi = 96,
 * Nr = 33 with four fields each way fits).  desc->flags must be 0
 * (KMHD_ERR_ARG otherwise).  Every call looks up the array's address on
 * desc->device, makes that device current for the call and makes the caller's
 * device current again before it returns.  All calls share the one array:
 * calls that overlap on the GPU (other host threads, other streams) race and
 * corrupt each other's results.
 * This entry point has no counterpart in the reference. */
int kmhd_sph_cycle_noalloc(const kmhd_sph_desc *desc, const double *d_rj_in, int64_t ld_in,
                           const int32_t *cols_b, double *d_rj_out, int64_t ld_out,
                           const int32_t *cols_f, void *stream);

/* Divergence of a flux vector's spectra, the step after the forward transform
 * that closes the u.grad(T) term (heat advection = -div(u T)): column
 * col_div = (dS/dr by the reference's radial FDM - dS/dr column) * max(g3, 1/2)
 * / r^2 for the vector in columns col_flux (S) and col_flux + 1 (dS/dr), with
 * fixed-field rows at the first and last radius, whose node values S are
 * replaced by fix_in[J] / fix_out[J] (NULL = zero).  Replaces
 * const_sph_scalar_advect with fixed-field boundaries
 * (MHD_src/sph_MHD/const_sph_divergence.f90:49-74: cal_sph_nod_vect_div2,
 * cal_sph_exp_rotation.f90:254-290; cal_sph_div_flux_4_fix_in / _fix_out,
 * cal_sph_exp_fixed_scalar.f90:381-456).  Needs Nr >= 3; host or device
 * pointers (ptr_kind). */
int kmhd_sph_div_flux(kmhd_sph *handle, double *d_rj, int64_t ld_rj, int32_t col_flux, int32_t col_div,
                      const double *fix_in, const double *fix_out, int32_t ptr_kind);

/* Curl of u x B, the induction term of the magnetic field equation: columns
 * col_rot .. col_rot + 2 = (pol, dpol/dr, tor) of the curl of the vector in
 * columns col_fld .. col_fld + 2 = (S, dS/dr, T): pol = T, dpol/dr = dT/dr and
 * tor = -d(dS/dr)/dr + l(l+1) S / r^2 by the reference's radial FDM, with
 * insulating boundaries (dpol/dr = (l+1) T / r at the first radius, -l T / r
 * at the last, tor = 0 there).  Replaces const_sph_rotation_uxb with
 * insulating boundaries (MHD_src/sph_MHD/const_sph_rotation.f90:167-187;
 * cal_sph_nod_vect_w_div_rot2, cal_sph_exp_rotation.f90:207-248;
 * cal_sph_nod_icb_ins_vp_rot2 / cal_sph_nod_cmb_ins_vp_rot2).  The column
 * ranges must not overlap; Nr >= 3; host or device pointers. */
int kmhd_sph_rot_induction(kmhd_sph *handle, double *d_rj, int64_t ld_rj, int32_t col_fld, int32_t col_rot,
                           int32_t ptr_kind);

/* Boundary conditions of a scalar (temperature, composition) for the
 * divergence of its flux: fixed field (the one-sided FDM row takes the
 * boundary value) or fixed flux (the row takes the given flux in place of the
 * derivative: cal_div_sph_in_fix_flux_2 / cal_div_sph_out_fix_flux_2,
 * MHD_src/sph_MHD/cal_sph_exp_fixed_flux.f90:134-157, 253-276); chosen as
 * sel_bc_sph_scalar_advect does (select_exp_scalar_bc.f90:219-277). */
#define KMHD_BC_FIXED_FIELD 0
#define KMHD_BC_FIXED_FLUX 1

/* kmhd_sph_div_flux with a boundary condition per side (KMHD_BC_FIXED_*):
 * val_in / val_out (J each, NULL = zero) are the fixed field or the fixed
 * flux spectra of that side. */
int kmhd_sph_div_flux_bc(kmhd_sph *handle, double *d_rj, int64_t ld_rj, int32_t col_flux, int32_t col_div,
                         int32_t bc_icb, int32_t bc_cmb, const double *val_in, const double *val_out,
                         int32_t ptr_kind);

/* Magnetic boundary conditions for the curl of u x B: insulator (as
 * kmhd_sph_rot_induction) or pseudo-vacuum, a purely radial field (pol = T,
 * dpol/dr = tor = 0: cal_sph_nod_icb_qvc_vp_rot2 / cal_sph_nod_cmb_qvc_vp_rot2,
 * MHD_src/sph_MHD/cal_sph_exp_nod_icb_qvac.f90:125-147,
 * cal_sph_exp_nod_cmb_qvac.f90:125-147); chosen as sel_bc_sph_rotation_uxb
 * does (select_exp_magne_bc.f90:222-262). */
#define KMHD_BC_INSULATOR 0
#define KMHD_BC_PSEUDO_VACUUM 1

int kmhd_sph_rot_induction_bc(kmhd_sph *handle, double *d_rj, int64_t ld_rj, int32_t col_fld, int32_t col_rot,
                              int32_t bc_icb, int32_t bc_cmb, int32_t ptr_kind);

/* Current density J = curl B from the magnetic field's spectra (columns
 * col_magne .. + 2) into col_current .. + 2 (the time loop's
 * const_grad_bp_and_current, const_sph_radial_grad.f90:166-200, forms the same
 * rows and also extends the potential field to radii outside the shell, which
 * a shell-only grid does not have).  Rows: pol = T, dpol/dr = dT/dr, tor =
 * -d2S/dr2 + l(l+1) S / r^2 with 3-point FDMs (cal_sph_nod_vect_rot2,
 * MHD_src/sph_MHD/cal_sph_exp_rotation.f90:157-203), boundary rows per
 * KMHD_BC_INSULATOR / KMHD_BC_PSEUDO_VACUUM: replaces const_sph_current
 * (const_sph_rotation.f90:141-158) with sel_bc_sph_current
 * (select_exp_magne_bc.f90:172-218).  The restart files hold B, not J. */
int kmhd_sph_current(kmhd_sph *handle, double *d_rj, int64_t ld_rj, int32_t col_magne, int32_t col_current,
                     int32_t bc_icb, int32_t bc_cmb, int32_t ptr_kind);

/* Velocity boundary conditions of the momentum equation (the reference's
 * iflag_icb / iflag_cmb for the velocity): non-slip and free slip. */
#define KMHD_BC_NON_SLIP 0
#define KMHD_BC_FREE_SLIP 1

/* Curl of a momentum force (advection, Lorentz force), the source of the
 * vorticity equation: as kmhd_sph_rot_induction in the interior; on each
 * boundary pol = T, dpol/dr = one-sided dT/dr and tor = -(d2S/dr2 - l(l+1)
 * S / r^2), with the two-point second derivative of the velocity condition
 * bc_icb / bc_cmb (KMHD_BC_*).  Replaces const_sph_force_rot2
 * (MHD_src/sph_MHD/const_sph_rotation.f90:225-250), called by
 * cal_rot_of_forces_sph_2 (cal_sph_field_by_rotation.f90:83-121), with the
 * rows of sel_bc_sph_vorticity (select_exp_velocity_bc.f90:215-262):
 * cal_sph_nod_icb_rigid_rot2 / cal_sph_nod_cmb_rigid_rot2
 * (set_sph_exp_rigid_ICB.f90:159-197, set_sph_exp_rigid_CMB.f90:129-166) and
 * cal_sph_nod_icb_free_rot2 / cal_sph_nod_cmb_free_rot2
 * (set_sph_exp_free_ICB.f90:131-166, set_sph_exp_free_CMB.f90).  The full-sphere
 * centre row and the rotating inner core's torque are not provided.  Column
 * ranges must not overlap; Nr >= 3; host or device pointers. */
int kmhd_sph_rot_force(kmhd_sph *handle, double *d_rj, int64_t ld_rj, int32_t col_fld, int32_t col_rot,
                       int32_t bc_icb, int32_t bc_cmb, int32_t ptr_kind);

/* Vorticity = curl u from the velocity's spectra into col_vort .. + 2, with
 * the interior rows of kmhd_sph_current and the velocity boundary rows of
 * kmhd_sph_rot_force (KMHD_BC_NON_SLIP / KMHD_BC_FREE_SLIP), as
 * const_sph_vorticity (MHD_src/sph_MHD/const_sph_rotation.f90:111-137).  The
 * time loop's const_grad_vp_and_vorticity (const_sph_radial_grad.f90:136-162,
 * called from cal_sol_sph_MHD_crank.f90) gives the same vorticity for a
 * velocity that meets its boundary condition; it also rewrites the velocity's
 * boundary values and its dS/dr column, which this call leaves alone.  The
 * restart files hold u, not the vorticity. */
int kmhd_sph_vorticity(kmhd_sph *handle, double *d_rj, int64_t ld_rj, int32_t col_velo, int32_t col_vort,
                       int32_t bc_icb, int32_t bc_cmb, int32_t ptr_kind);

/* Divergence of a momentum force (the pressure equation's source): as
 * kmhd_sph_div_flux with each boundary node's own S in the one-sided rows.
 * Replaces const_sph_div_force (MHD_src/sph_MHD/const_sph_divergence.f90:79-108:
 * cal_sph_nod_vect_div2, cal_sph_nod_nobc_in_div2 / _out_div2,
 * cal_sph_exp_nod_none_bc.f90:153-185, 309-341). */
int kmhd_sph_div_force(kmhd_sph *handle, double *d_rj, int64_t ld_rj, int32_t col_fld, int32_t col_div,
                       int32_t ptr_kind);

/* Curl of the radial buoyancy, the toroidal source of the vorticity equation:
 * column col_out = coef_t * T * r, or (coef_t * T + coef_c * C) * r when
 * col_c >= 0 (thermal and compositional buoyancy).  Replaces
 * cal_rot_radial_self_gravity (MHD_src/sph_MHD/cal_rot_buoyancies_sph_MHD.f90:46-165,
 * called from cal_sol_sph_MHD_crank.f90) into itor%i_rot_buoyancy.  Host or
 * device pointers. */
int kmhd_sph_rot_buoyancy(kmhd_sph *handle, double *d_rj, int64_t ld_rj, int32_t col_t, double coef_t,
                          int32_t col_c, double coef_c, int32_t col_out, int32_t ptr_kind);

/* Curl of the Coriolis term for a rotation about z, formed in spectral space
 * from the velocity (columns col_velo .. col_velo + 2 = S, dS/dr, T) and the
 * vorticity (col_vort .. col_vort + 2): column col_out = poloidal and
 * col_out + 2 = toroidal part of curl(-coef_cor z x u) by the Adams-Gaunt and
 * Elsasser couplings of each mode to (l-1, m), (l+1, m) and (l, -m); column
 * col_out + 1 is not written.  Replaces sum_coriolis_rlm with a fixed inner
 * core (MHD_src/sph_MHD/t_coriolis_terms_rlm.f90:190-292:
 * sum_rot_coriolis_rlm_10, sum_coriolis_terms_rlm.f90:94-189; the tables of
 * init_sum_coriolis_rlm, interact_coriolis_rlm.f90) and the copy into the
 * forward transform's output (copy_coriolis_terms_rlm).  The two written
 * columns may not be input columns; host or device pointers. */
int kmhd_sph_rot_coriolis(kmhd_sph *handle, double *d_rj, int64_t ld_rj, int32_t col_velo, int32_t col_vort,
                          int32_t col_out, double coef_cor, int32_t ptr_kind);

/* Makes every following kmhd_sph_cycle / kmhd_sph_batch_cycle of the handle
 * also write the curl of the Coriolis term, as the reference's
 * sph_b_trans_w_coriolis / sph_f_trans_w_coriolis do (sum_coriolis_rlm on the
 * received spectra, copy_coriolis_terms_rlm into the forward output;
 * MHD_src/sph_MHD/sph_trans_w_coriols.f90:113-246): the velocity and vorticity
 * are backward vector fields iv_velo and iv_vort (0-based among the nvector_b
 * vectors, read through that call's cols_b); the poloidal part goes to output
 * column col_out and the toroidal part to col_out + 2 of d_rj_out (col_out + 1
 * is not written).  With host pointers the inputs are read from the cycle's
 * own staged copies (no second transfer).  The two columns may not be written
 * by a forward field, nor be input columns when input and output are one
 * array (KMHD_ERR_ARG at the cycle call).  iv_velo < 0 switches it off.  The
 * tables are built here (device memory), not inside the cycle.  The separable
 * calls split it as the reference does: kmhd_sph_b_trans forms the curl from
 * its input spectra and the next kmhd_sph_f_trans writes it into d_rj's
 * columns col_out and col_out + 2. */
int kmhd_sph_set_coriolis(kmhd_sph *handle, double coef_cor, int32_t iv_velo, int32_t iv_vort, int32_t col_out);

/* Backward transform at the poles, for grids with pole points: v_pole is a
 * (2 Nr) x ncomp_b column-major array, row k the north pole and row Nr + k the
 * south pole of radius k; scalars as values, vectors in Cartesian components
 * (x, y, z; z is the radial direction at the north pole and its opposite at the
 * south pole), from the orders 0 and +-1 of the spectra in columns cols_b
 * (as kmhd_sph_b_trans).  Replaces pole_backward_transforms without the centre
 * point (PARALLEL_src/SPH_SHELL_src/pole_sph_transform.f90:107-162:
 * schmidt_b_trans_pole_vect / _scalar, schmidt_b_trans_at_pole.f90:88-289).
 * Host or device pointers (both arrays the same kind). */
int kmhd_sph_b_trans_pole(kmhd_sph *handle, const double *d_rj, int64_t ld_rj, const int32_t *cols_b, double *v_pole,
                          int32_t ptr_kind);

/* Backward transform at the centre of a full-sphere grid (the r = 0 node of a
 * mesh with a centre point): v_center[0 .. ncomp_b) holds that node's
 * components in the order of v_pole; for every backward vector, from the
 * poloidal column S at the innermost radius r_1 = radius[0]:
 * v[3f] = -2 S(1,-1) / r_1^2, v[3f+1] = -2 S(1,+1) / r_1^2, v[3f+2] =
 * 2 S(1,0) / r_1^2.  Scalar entries are not written (the reference leaves
 * them unchanged).  Replaces schmidt_b_trans_center_vect / _scalar
 * (PARALLEL_src/SPH_SHELL_src/schmidt_b_trans_at_center.f90:45-119), called
 * by pole_backward_transforms for iflag_MESH_w_center
 * (pole_sph_transform.f90:148-157).  Host or device pointers (both arrays
 * the same kind). */
int kmhd_sph_b_trans_center(kmhd_sph *handle, const double *d_rj, int64_t ld_rj, const int32_t *cols_b,
                            double *v_center, int32_t ptr_kind);

/* Legendre path the handle runs: 1 = the tier's split path, 0 = FP64 DMMA
 * (FP64 tier, or a split-tier handle the autotuner moved to FP64). */
int kmhd_sph_get_path(const kmhd_sph *handle, int32_t *path);

/* Legendre path (as kmhd_sph_get_path), slice products per GEMM of the split
 * path (26 or 21 split, 10 or 6 fp32acc, 0 for the FP64 tier), and after an
 * autotuned batch call the candidates' cycle times (ms3: FP64 path, full and
 * reduced product count) and errors against the FP64 path (err3; 0 for the
 * FP64 candidate); zeros before tuning.  Any pointer may be NULL.  Extends the
 * reference's start-up choice of a Legendre variant (init_sphrical_transform_MHD.f90:201-345). */
int kmhd_sph_get_tuning(const kmhd_sph *handle, int32_t *path, int32_t *products, float *ms3, double *err3);

/* Pins the slice products per GEMM of a split-tier handle: 26 or 21 (split),
 * 10 or 6 (fp32acc); KMHD_ERR_ARG otherwise.  21 (6) drops the digit pairs of
 * the highest group: about 20% (40%) fewer tensor-core products, an error
 * near 256 times larger.  No counterpart in the reference. */
int kmhd_sph_set_products(kmhd_sph *handle, int32_t products);

/* Device bytes held by the handle. */
int64_t kmhd_sph_device_bytes(const kmhd_sph *handle);

const char *kmhd_strerror(int status);

/* Failure-path self-test (no counterpart in the reference): runs one of the
 * library's bounded device waits -- which = 0 the tcgen05 pipeline's mbarrier
 * wait, 1 the FFT's staging wait -- on an mbarrier that nothing completes.
 * The wait runs out (2^16 wait rounds, well under a second), the kernel records
 * KMHD_ERR_TIMEOUT in a device error word and returns, and the call returns
 * that status; the CUDA context stays usable.  No GPU fault is involved. */
int kmhd_selftest_wait_timeout(int device, int which);

#ifdef __cplusplus
}
#endif

#endif /* KMHD_SPH_H */
