// Drives the C++ mirror like the reference's MHD loop does: one d_fld array
// holding velocity, vorticity, magnetic field, temperature and the forces, the
// transform segment of nonlinear_by_pseudo_sph applied in place, compared with
// the CPU FP64 oracle (test infrastructure) on the same columns.
#include <dlfcn.h>

#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "../../kemorin_mhd_b200/host/sph_trans_4_MHD.hpp"

using namespace kmhd::calypso;

// Second mode (an output path as the third argument): the full MHD field set
// through the spectral steps around the transform, as the reference's time
// step orders them -- const_grad_vp_and_vorticity / const_grad_bp_and_current,
// the cycle with the Coriolis curl, rot_momentum_eq_exp_sph,
// cal_rot_radial_self_gravity -- on host arrays; d_fld is written to the path
// (nnod x 47 doubles, column-major) for the test to compare with the oracle.
static int run_full(int tier, const char* out_path) {
  const int L = 15, nth = 24, nph = 48, nr = 6;
  std::vector<double> radius(nr);
  for (int k = 0; k < nr; ++k)
    radius[k] = 0.35 / 0.65 + 0.5 * (1.0 / 0.65 - 0.35 / 0.65) * (1.0 - std::cos(M_PI * k / (nr - 1)));
  PhysAddress ipol;
  ipol.i_velo = 1; ipol.i_vort = 4; ipol.i_magne = 7; ipol.i_current = 10; ipol.i_temp = 13; ipol.i_light = 14;
  ipol.i_m_advect = 15; ipol.i_lorentz = 18; ipol.i_vp_induct = 21; ipol.i_h_flux = 24; ipol.i_c_flux = 27;
  ipol.i_k_heli = 30;
  ipol.i_rot_inertia = 31; ipol.i_rot_Lorentz = 34; ipol.i_induction = 37; ipol.i_h_advect = 40;
  ipol.i_c_advect = 41; ipol.i_rot_Coriolis = 42; ipol.i_rot_buoyancy = 45;
  const int ntot = 47;
  const long J = (long)(L + 1) * (L + 1), nnod = J * nr;
  std::vector<double> d_fld(nnod * ntot, 0.0);
  std::mt19937_64 g(11);
  std::normal_distribution<double> nd;
  for (int c : {0, 1, 2, 6, 7, 8, 12, 13})
    for (long i = 0; i < nnod; ++i) d_fld[c * nnod + i] = nd(g);
  try {
    SphTransMHD tr(L, nth, nph, radius, ipol, tier);
    SphBoundaries bc;   // non-slip, insulating, fixed (zero) temperature and composition
    tr.init_sum_coriolis_rlm(2.0e2);
    tr.const_grad_vp_and_vorticity(d_fld.data(), bc);
    tr.const_grad_bp_and_current(d_fld.data(), bc);
    tr.nonlinear_by_pseudo_sph(d_fld.data());
    tr.rot_momentum_eq_exp_sph(d_fld.data(), bc);
    tr.cal_rot_radial_self_gravity(d_fld.data(), 3.0, -1.5);
  } catch (const TransformError& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 3;
  }
  FILE* f = std::fopen(out_path, "wb");
  if (!f) return 2;
  const size_t n = std::fwrite(d_fld.data(), sizeof(double), d_fld.size(), f);
  std::fclose(f);
  return n == d_fld.size() ? 0 : 2;
}

int main(int argc, char** argv) {
  if (argc < 2) { std::fprintf(stderr, "usage: %s liboracle.so [tier [out]]\n", argv[0]); return 2; }
  if (argc > 3) return run_full(std::atoi(argv[2]), argv[3]);
  const int L = 15, nth = 24, nph = 48, nr = 5;
  std::vector<double> radius(nr);
  for (int k = 0; k < nr; ++k)
    radius[k] = 0.35 / 0.65 + 0.5 * (1.0 / 0.65 - 0.35 / 0.65) * (1.0 - std::cos(M_PI * k / (nr - 1)));
  PhysAddress ipol;
  ipol.i_velo = 1; ipol.i_vort = 4; ipol.i_magne = 7; ipol.i_temp = 10;
  ipol.i_m_advect = 11; ipol.i_vp_induct = 14; ipol.i_h_flux = 17; ipol.i_k_heli = 20;
  const int ntot = 20;
  const long J = (long)(L + 1) * (L + 1), nnod = J * nr;
  std::vector<double> d_fld(nnod * ntot, 0.0);
  std::mt19937_64 g(7);
  std::normal_distribution<double> nd;
  for (long i = 0; i < nnod * 10; ++i) d_fld[i] = nd(g);
  try {
    SphTransMHD tr(L, nth, nph, radius, ipol, argc > 2 ? std::atoi(argv[2]) : KMHD_TIER_FP64);
    std::vector<double> in(d_fld);
    tr.nonlinear_by_pseudo_sph(d_fld.data());
    // oracle
    void* so = dlopen(argv[1], RTLD_NOW);
    if (!so) { std::fprintf(stderr, "%s\n", dlerror()); return 2; }
    typedef void* (*create_t)(int, int, int, int, const double*, int, int, int, int, int, const int*, const int*,
                              const int*, const double*, int);
    typedef void (*cycle_t)(void*, const double*, long long, const int*, double*, long long, const int*);
    auto create = (create_t)dlsym(so, "oracle_create");
    auto cycle = (cycle_t)dlsym(so, "oracle_cycle");
    const auto& a = tr.addresses();
    std::vector<int> kind, pa, pb;
    std::vector<double> cf;
    for (auto& p : a.products) { kind.push_back(p.kind); pa.push_back(p.a); pb.push_back(p.b); cf.push_back(p.coef); }
    void* o = create(L, nth, nph, nr, radius.data(), a.nvector_b, a.nscalar_b, a.nvector_f, a.nscalar_f,
                     (int)kind.size(), kind.data(), pa.data(), pb.data(), cf.data(), 2);
    std::vector<int> cb(a.cols_b.begin(), a.cols_b.end()), cfo(a.cols_f.begin(), a.cols_f.end());
    std::vector<double> ref(nnod * ntot, 0.0);
    cycle(o, in.data(), nnod, cb.data(), ref.data(), nnod, cfo.data());
    double worst = 0.0;
    for (int c = 10; c < ntot; ++c) {
      double e = 0.0, m = 0.0;
      for (long i = 0; i < nnod; ++i) {
        e = std::fmax(e, std::fabs(d_fld[c * nnod + i] - ref[c * nnod + i]));
        m = std::fmax(m, std::fabs(ref[c * nnod + i]));
      }
      worst = std::fmax(worst, e / m);
    }
    std::printf("max relative error vs oracle: %.3e\n", worst);
    return worst <= 1e-12 ? 0 : 1;
  } catch (const TransformError& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 3;
  }
}
