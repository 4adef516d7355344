// sph_trans_4_MHD.hpp -- C++ host mirror of the reference's MHD transform
// entry points, layered on the C-ABI of include/kmhd_sph.h.
//
// Names and argument meaning follow the reference's Fortran interface:
//   sph_back_trans_4_MHD   (MHD_src/sph_MHD/sph_transforms_4_MHD.f90:88)
//   sph_forward_trans_4_MHD (MHD_src/sph_MHD/sph_transforms_4_MHD.f90:137)
//   nonlinear_by_pseudo_sph (MHD_src/sph_MHD/cal_nonlinear.f90:118), transform segment
// with the same data: rj_fld%d_fld(nnod_rj, ntot_phys) column-major, field
// addresses ipol%i_* as 1-based column numbers (0 = field absent), and the
// grid fields fld_rtp(nnod_rtp, ncomp_rj_2_rtp) / frc_rtp(nnod_rtp,
// ncomp_rtp_2_rj).  The reference aborts through calypso_MPI_abort on error;
// this layer throws kmhd::calypso::TransformError carrying the C-ABI status.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/kmhd_sph.h"

namespace kmhd {
namespace calypso {

struct TransformError : std::runtime_error {
  int status;
  TransformError(int st, const std::string& where)
      : std::runtime_error(where + ": " + kmhd_strerror(st)), status(st) {}
};

inline void check(int st, const char* where) {
  if (st != KMHD_OK) throw TransformError(st, where);
}

// phys_address subset used by the transform and the spectral steps around it
// (1-based columns of d_fld, 0 = absent; ipol% addresses: the poloidal column
// of a vector, whose dS/dr and toroidal columns follow)
struct PhysAddress {
  int i_velo = 0, i_vort = 0, i_magne = 0, i_current = 0;                // rj -> rtp vectors
  int i_temp = 0, i_light = 0;                                            // rj -> rtp scalars
  int i_m_advect = 0, i_lorentz = 0, i_vp_induct = 0, i_h_flux = 0;       // rtp -> rj vectors
  int i_c_flux = 0, i_k_heli = 0;                                         // (u C), (u . omega)
  // spectral results of rot_momentum_eq_exp_sph / the Coriolis and buoyancy terms
  int i_rot_inertia = 0, i_rot_Lorentz = 0, i_induction = 0, i_h_advect = 0, i_c_advect = 0;
  int i_rot_Coriolis = 0, i_rot_buoyancy = 0;
};

// Boundary conditions of the spectral steps (sph_bc_U, sph_bc_B, sph_bc_T, sph_bc_C)
struct SphBoundaries {
  int velo_icb = KMHD_BC_NON_SLIP, velo_cmb = KMHD_BC_NON_SLIP;
  int magne_icb = KMHD_BC_INSULATOR, magne_cmb = KMHD_BC_INSULATOR;
  int temp_icb = KMHD_BC_FIXED_FIELD, temp_cmb = KMHD_BC_FIXED_FIELD;
  const double *temp_icb_val = nullptr, *temp_cmb_val = nullptr;   // ICB_fld / ICB_flux spectra (J), NULL = 0
  int comp_icb = KMHD_BC_FIXED_FIELD, comp_cmb = KMHD_BC_FIXED_FIELD;
  const double *comp_icb_val = nullptr, *comp_cmb_val = nullptr;
};

// Transform addresses built like b_trans_address_* / f_trans_address_*
// (MHD_src/sph_MHD/set_address_sph_trans_MHD.f90): vectors first, then scalars.
struct TransAddresses {
  std::vector<int32_t> cols_b, cols_f;   // 0-based first columns per field
  int nvector_b = 0, nscalar_b = 0, nvector_f = 0, nscalar_f = 0;
  std::vector<kmhd_product> products;
};

inline TransAddresses set_addresses_trans_sph_MHD(const PhysAddress& ipol) {
  TransAddresses t;
  int iv_velo = -1, iv_vort = -1, iv_magne = -1, iv_current = -1, is_temp = -1, is_light = -1;
  auto addv = [&](int col, int& slot) { if (col > 0) { slot = t.nvector_b++; t.cols_b.push_back(col - 1); } };
  addv(ipol.i_velo, iv_velo);
  addv(ipol.i_vort, iv_vort);
  addv(ipol.i_magne, iv_magne);
  addv(ipol.i_current, iv_current);
  if (ipol.i_temp > 0) { is_temp = t.nscalar_b++; t.cols_b.push_back(ipol.i_temp - 1); }
  if (ipol.i_light > 0) { is_light = t.nscalar_b++; t.cols_b.push_back(ipol.i_light - 1); }
  if (ipol.i_m_advect > 0 && iv_vort >= 0 && iv_velo >= 0) {     // omega x u
    t.products.push_back({KMHD_PROD_CROSS, iv_vort, iv_velo, 1.0});
    t.cols_f.push_back(ipol.i_m_advect - 1); ++t.nvector_f;
  }
  if (ipol.i_lorentz > 0 && iv_current >= 0 && iv_magne >= 0) {  // J x B
    t.products.push_back({KMHD_PROD_CROSS, iv_current, iv_magne, 1.0});
    t.cols_f.push_back(ipol.i_lorentz - 1); ++t.nvector_f;
  }
  if (ipol.i_vp_induct > 0 && iv_velo >= 0 && iv_magne >= 0) {   // u x B
    t.products.push_back({KMHD_PROD_CROSS, iv_velo, iv_magne, 1.0});
    t.cols_f.push_back(ipol.i_vp_induct - 1); ++t.nvector_f;
  }
  if (ipol.i_h_flux > 0 && iv_velo >= 0 && is_temp >= 0) {       // u T
    t.products.push_back({KMHD_PROD_VEC_SCALAR, iv_velo, is_temp, 1.0});
    t.cols_f.push_back(ipol.i_h_flux - 1); ++t.nvector_f;
  }
  if (ipol.i_c_flux > 0 && iv_velo >= 0 && is_light >= 0) {      // u C
    t.products.push_back({KMHD_PROD_VEC_SCALAR, iv_velo, is_light, 1.0});
    t.cols_f.push_back(ipol.i_c_flux - 1); ++t.nvector_f;
  }
  if (ipol.i_k_heli > 0 && iv_velo >= 0 && iv_vort >= 0) {       // u . omega
    t.products.push_back({KMHD_PROD_DOT, iv_velo, iv_vort, 1.0});
    t.cols_f.push_back(ipol.i_k_heli - 1); ++t.nscalar_f;
  }
  return t;
}

// One transform instance (the reference's sph / trans_p / WK_sph state).
class SphTransMHD {
 public:
  SphTransMHD(int l_truncation, int nth_rtm, int nph_rtp, const std::vector<double>& radius_1d_rj_r,
              const PhysAddress& ipol, int tier = KMHD_TIER_FP64, int device = 0)
      : ipol_(ipol), addr_(set_addresses_trans_sph_MHD(ipol)), nr_(static_cast<int>(radius_1d_rj_r.size())),
        nnod_rj_((int64_t)(l_truncation + 1) * (l_truncation + 1) * radius_1d_rj_r.size()) {
    kmhd_sph_desc d = {};
    d.ltr = l_truncation;
    d.nth = nth_rtm;
    d.nph = nph_rtp;
    d.nr = nr_;
    d.radius = radius_1d_rj_r.data();
    d.nvector_b = addr_.nvector_b;
    d.nscalar_b = addr_.nscalar_b;
    d.nvector_f = addr_.nvector_f;
    d.nscalar_f = addr_.nscalar_f;
    d.nproduct = static_cast<int32_t>(addr_.products.size());
    d.products = addr_.products.data();
    d.tier = tier;
    d.device = device;
    check(kmhd_sph_create(&d, &h_), "initialize_sph_trans");
  }
  ~SphTransMHD() { if (h_) kmhd_sph_destroy(h_); }
  SphTransMHD(const SphTransMHD&) = delete;
  SphTransMHD& operator=(const SphTransMHD&) = delete;

  const TransAddresses& addresses() const { return addr_; }

  // rj_fld%d_fld (host, nnod_rj x ntot_phys) -> fld_rtp (host, nnod_rtp x ncomp_rj_2_rtp)
  void sph_back_trans_4_MHD(const double* d_fld, double* fld_rtp) {
    check(kmhd_sph_b_trans(h_, d_fld, nnod_rj_, addr_.cols_b.data(), fld_rtp, KMHD_PTR_HOST),
          "sph_back_trans_4_MHD");
  }
  // frc_rtp (host, nnod_rtp x ncomp_rtp_2_rj) -> rj_fld%d_fld forces
  void sph_forward_trans_4_MHD(const double* frc_rtp, double* d_fld) {
    check(kmhd_sph_f_trans(h_, frc_rtp, d_fld, nnod_rj_, addr_.cols_f.data(), KMHD_PTR_HOST),
          "sph_forward_trans_4_MHD");
  }
  // backward transform -> nonlinear_terms_in_rtp -> forward transform, in place on d_fld
  // (with the curl of the Coriolis term when init_sum_coriolis_rlm was called)
  void nonlinear_by_pseudo_sph(double* d_fld) {
    check(kmhd_sph_cycle(h_, d_fld, nnod_rj_, addr_.cols_b.data(), d_fld, nnod_rj_, addr_.cols_f.data(),
                         KMHD_PTR_HOST),
          "nonlinear_by_pseudo_sph");
  }

  // init_sum_coriolis_rlm (t_coriolis_terms_rlm.f90): the cycle also writes the
  // curl of -coef_cor z x u into ipol%i_rot_Coriolis / itor%i_rot_Coriolis
  void init_sum_coriolis_rlm(double coef_cor) {
    int iv = -1, iw = -1, n = 0;
    if (ipol_.i_velo > 0) iv = n++;
    if (ipol_.i_vort > 0) iw = n++;
    if (iv < 0 || iw < 0 || ipol_.i_rot_Coriolis <= 0) throw TransformError(KMHD_ERR_ARG, "init_sum_coriolis_rlm");
    check(kmhd_sph_set_coriolis(h_, coef_cor, iv, iw, ipol_.i_rot_Coriolis - 1), "init_sum_coriolis_rlm");
  }

  // const_grad_vp_and_vorticity / const_grad_bp_and_current
  // (MHD_src/sph_MHD/const_sph_radial_grad.f90:136-200): omega = curl u and
  // J = curl B from the spectra, before the backward transform
  void const_grad_vp_and_vorticity(double* d_fld, const SphBoundaries& bc) {
    if (ipol_.i_velo > 0 && ipol_.i_vort > 0)
      check(kmhd_sph_vorticity(h_, d_fld, nnod_rj_, ipol_.i_velo - 1, ipol_.i_vort - 1, bc.velo_icb, bc.velo_cmb,
                               KMHD_PTR_HOST),
            "const_grad_vp_and_vorticity");
  }
  void const_grad_bp_and_current(double* d_fld, const SphBoundaries& bc) {
    if (ipol_.i_magne > 0 && ipol_.i_current > 0)
      check(kmhd_sph_current(h_, d_fld, nnod_rj_, ipol_.i_magne - 1, ipol_.i_current - 1, bc.magne_icb,
                             bc.magne_cmb, KMHD_PTR_HOST),
            "const_grad_bp_and_current");
  }

  // rot_momentum_eq_exp_sph (MHD_src/sph_MHD/cal_sph_field_by_rotation.f90:49-78)
  // after the forward transform: the curls of the advection and the Lorentz
  // force (cal_rot_of_forces_sph_2), the induction (cal_rot_of_induction_sph),
  // and the heat and composition advection (cal_div_of_fluxes_sph)
  void rot_momentum_eq_exp_sph(double* d_fld, const SphBoundaries& bc) {
    const int64_t ld = nnod_rj_;
    if (ipol_.i_m_advect > 0 && ipol_.i_rot_inertia > 0)
      check(kmhd_sph_rot_force(h_, d_fld, ld, ipol_.i_m_advect - 1, ipol_.i_rot_inertia - 1, bc.velo_icb,
                               bc.velo_cmb, KMHD_PTR_HOST),
            "cal_rot_of_forces_sph_2 (advection)");
    if (ipol_.i_lorentz > 0 && ipol_.i_rot_Lorentz > 0)
      check(kmhd_sph_rot_force(h_, d_fld, ld, ipol_.i_lorentz - 1, ipol_.i_rot_Lorentz - 1, bc.velo_icb,
                               bc.velo_cmb, KMHD_PTR_HOST),
            "cal_rot_of_forces_sph_2 (Lorentz)");
    if (ipol_.i_vp_induct > 0 && ipol_.i_induction > 0)
      check(kmhd_sph_rot_induction_bc(h_, d_fld, ld, ipol_.i_vp_induct - 1, ipol_.i_induction - 1, bc.magne_icb,
                                      bc.magne_cmb, KMHD_PTR_HOST),
            "cal_rot_of_induction_sph");
    if (ipol_.i_h_flux > 0 && ipol_.i_h_advect > 0)
      check(kmhd_sph_div_flux_bc(h_, d_fld, ld, ipol_.i_h_flux - 1, ipol_.i_h_advect - 1, bc.temp_icb, bc.temp_cmb,
                                 bc.temp_icb_val, bc.temp_cmb_val, KMHD_PTR_HOST),
            "cal_div_of_fluxes_sph (heat)");
    if (ipol_.i_c_flux > 0 && ipol_.i_c_advect > 0)
      check(kmhd_sph_div_flux_bc(h_, d_fld, ld, ipol_.i_c_flux - 1, ipol_.i_c_advect - 1, bc.comp_icb, bc.comp_cmb,
                                 bc.comp_icb_val, bc.comp_cmb_val, KMHD_PTR_HOST),
            "cal_div_of_fluxes_sph (composition)");
  }

  // cal_rot_radial_self_gravity (MHD_src/sph_MHD/cal_rot_buoyancies_sph_MHD.f90:46-101)
  void cal_rot_radial_self_gravity(double* d_fld, double coef_buo, double coef_comp_buo) {
    if (ipol_.i_rot_buoyancy <= 0 || ipol_.i_temp <= 0) return;
    // into itor%i_rot_buoyancy, the vector's toroidal column
    check(kmhd_sph_rot_buoyancy(h_, d_fld, nnod_rj_, ipol_.i_temp - 1, coef_buo,
                                ipol_.i_light > 0 ? ipol_.i_light - 1 : -1, coef_comp_buo,
                                ipol_.i_rot_buoyancy - 1 + 2, KMHD_PTR_HOST),
          "cal_rot_radial_self_gravity");
  }

 private:
  PhysAddress ipol_;
  TransAddresses addr_;
  int nr_;
  int64_t nnod_rj_;
  kmhd_sph* h_ = nullptr;
};

}  // namespace calypso
}  // namespace kmhd
