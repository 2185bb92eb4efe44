// A C++23 caller of the reference's src/physics Kerr API, compiled against
// include/bh_physics_compat.hpp and linked with libblackhole_b200.so only.
//
//   physics_compat_main info                      no GPU call: the pure helpers
//   physics_compat_main potentials IN OUT         kerrPotentials per element
//   physics_compat_main step IN OUT               kerrStepMino, 1 step, each element
//   physics_compat_main trace IN OUT              KerrRaytracer::trace (batched span form,
//                                                 then element 0 with the path recorded)
// IN and OUT are raw little-endian float64 files (layouts in test_physics_compat.py).
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <span>
#include <string>
#include <vector>

#include "bh_physics_compat.hpp"

namespace {

std::vector<double> read_all(const char* path) {
  std::ifstream f(path, std::ios::binary);
  std::vector<char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  std::vector<double> v(b.size() / sizeof(double));
  std::memcpy(v.data(), b.data(), v.size() * sizeof(double));
  return v;
}

void write_all(const char* path, const std::vector<double>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(double)));
}

}  // namespace

int main(int argc, char** argv) {
  using namespace physics;
  const std::string mode = argc > 1 ? argv[1] : "info";
  try {
    if (mode == "info") {
      const KerrGeodesicConsts c = kerrEquatorialConsts(5.0, 2.0);
      const KerrGeodesicState s = kerrEquatorialState(30.0, 0.25, -0.5);
      std::printf("%.17g %.17g %.17g %.17g %.17g %.17g\n", c.e, c.lz, c.q, s.theta, s.signR, s.signTheta);
      return 0;
    }
    if (argc < 4) {
      std::fprintf(stderr, "usage: %s MODE IN OUT\n", argv[0]);
      return 2;
    }
    const std::vector<double> in = read_all(argv[2]);
    std::vector<double> out;
    if (mode == "potentials" || mode == "step") {
      // n, mass, a, then [n] r, theta, phi, t, signR, signTheta, e, lz, q, dlam
      const size_t n = size_t(in[0]);
      const double mass = in[1], a = in[2];
      const double* col = in.data() + 3;
      auto at = [&](int k, size_t i) { return col[k * n + i]; };
      for (size_t i = 0; i < n; ++i) {
        const KerrGeodesicConsts c{at(6, i), at(7, i), at(8, i)};
        if (mode == "potentials") {
          const KerrPotentials p = kerrPotentials(at(0, i), at(1, i), mass, a, c);
          out.insert(out.end(), {p.rPot, p.dRdr, p.thetaPot, p.dThetadtheta});
        } else {
          const KerrGeodesicState s{at(0, i), at(1, i), at(2, i), at(3, i), at(4, i), at(5, i)};
          const KerrGeodesicState t = kerrStepMino(s, mass, a, c, at(9, i));
          out.insert(out.end(), {t.r, t.theta, t.phi, t.t, t.signR, t.signTheta});
        }
      }
    } else if (mode == "trace") {
      // n, mass, spin parameter, step, max_steps, r_escape, then [n] state (6), consts (3)
      const size_t n = size_t(in[0]);
      KerrRaytracer tr(in[1], in[2]);
      tr.setStepSize(in[3]);
      tr.setMaxSteps(int(in[4]));
      tr.setEscapeRadius(in[5]);
      const double* col = in.data() + 6;
      std::vector<KerrGeodesicState> st(n);
      std::vector<KerrGeodesicConsts> cs(n);
      for (size_t i = 0; i < n; ++i) {
        st[i] = {col[i], col[n + i], col[2 * n + i], col[3 * n + i], col[4 * n + i], col[5 * n + i]};
        cs[i] = {col[6 * n + i], col[7 * n + i], col[8 * n + i]};
      }
      const std::vector<RayTraceResult> res = tr.trace(std::span<const KerrGeodesicState>(st),
                                                       std::span<const KerrGeodesicConsts>(cs));
      for (const RayTraceResult& r : res)
        out.insert(out.end(), {double(int(r.status)), double(r.stepsTaken), r.totalDistance, r.finalPosition.x,
                               r.finalPosition.y, r.finalPosition.z, r.redshift});
      tr.setRecordPath(true);
      const RayTraceResult one = tr.trace(st[0], cs[0]);
      out.insert(out.end(), {double(int(one.status)), double(one.stepsTaken), one.totalDistance,
                             one.finalPosition.x, one.finalPosition.y, one.finalPosition.z, one.redshift,
                             double(one.path.size())});
    } else {
      std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
      return 2;
    }
    write_all(argv[3], out);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
