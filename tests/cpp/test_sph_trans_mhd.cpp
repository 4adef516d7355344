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

int main(int argc, char** argv) {
  if (argc < 2) { std::fprintf(stderr, "usage: %s liboracle.so\n", argv[0]); return 2; }
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
