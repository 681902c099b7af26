// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// CPU oracle for the DFSPH liquid step of argonrobotics-ai/alloy (alloy/solvers/sph), restated in plain C++ from
// the reference's Warp kernels. Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may load it, and there
// only as the checker or the timed CPU baseline; the CUDA product never links or calls it.
//
// What it follows (reference file:line, paths inside the alloy project):
//   kernels.py:41-77      cubic / Wendland W and grad W              -> wf()
//   kernels.py:80-138     projected kernel, half-space volume Psi    -> halfspace()
//   neighbors.py:36-51    particle groups (fluid = world, wall = -2 - world)
//   neighbors.py:160-195  id-sorted lists, lowest K kept, overflow   -> build_lists()
//   particle_walls.py:65-119  wall colour, 30-step bisection, plane  -> wall_slots()
//   boundary.py:190-396, boundary_slots.py:13-108  up to four slots per particle: static box walls (newton
//                          geometry/kernels.py:310-370 box SDF) and the particle wall, nearest first, duplicate
//                          eviction, fit and taper, inclusion-exclusion            -> wall_slots()
//   pressure.py:144-193   density and DFSPH factor                   -> density_alpha()
//   pressure.py:196-261   density rate, solve source, warm start     -> solve_init()
//   pressure.py:264-352   pressure acceleration, relaxed Jacobi      -> accel(), jacobi()
//   pressure.py:355-390   per-world start and stop test              -> solve()
//   pressure.py:393-480   lone-particle limit, apply pressure, lone-particle wall friction
//   solve_driver.py:121-186  solve orchestration (Jacobi branch)
//   reduce.py:185-227     per-world float64 sums and max             -> world_sum() (tree order below)
//   integrate.py:60-326   XSPH, advection, projection onto walls and particle walls, sweep past fast steps, speed
//   particle_walls.py:131-135  wall particles advance with their own velocity
//   emitters.py:67-164    layer emitters, sinks and escape box, int64 mass ledger
//   solver.py:218-268     step order
//
// Arithmetic contract. The FP32 instantiation evaluates every expression in a fixed order with explicit fused
// multiply-adds (std::fma) and correctly rounded sqrt and division, compiled with -ffp-contract=off, so that the
// CUDA kernels (same order, __fmaf_rn, -fmad=false) reproduce it bit for bit. Pair distances use the unfused
// (dx*dx + dy*dy) + dz*dz, the reference's dot. Neighbour sums run in ascending particle id (the reference's order);
// wall-colour sums run in ascending wall-particle id (the reference sums in hash-grid visit order, which Warp does
// not pin). Per-world float64 sums use the tree order documented at world_sum(). The FP64 instantiation runs the
// same algorithm in double for error reports.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int FLAG_ACTIVE = 1;  // newton ParticleFlags.ACTIVE (geometry/flags.py:14)
constexpr int PROJECT_PASSES = 4;  // integrate.py:50
constexpr int NS = 4;              // boundary slots per particle (boundary.py:36)
constexpr float COS_SAME = 0.85f;  // boundary_slots.py:9
constexpr int BISECT = 30;         // particle_walls.py:44
constexpr double C_MIN = 1.0e-4;   // particle_walls.py:43

inline float fma_(float a, float b, float c) { return std::fmaf(a, b, c); }
inline double fma_(double a, double b, double c) { return std::fma(a, b, c); }
template <class R> inline R maxr(R a, R b) { return a > b ? a : b; }
template <class R> inline R minr(R a, R b) { return a < b ? a : b; }
template <class R> inline R clampr(R x, R lo, R hi) { return minr(maxr(x, lo), hi); }

template <class R> struct V3 { R x, y, z; };
template <class R> inline V3<R> sub(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
// the reference's dot (left to right, unfused); used for pair distances
template <class R> inline R dot_plain(V3<R> a, V3<R> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
// fused dot used everywhere else
template <class R> inline R dotf(V3<R> a, V3<R> b) { return fma_(a.z, b.z, fma_(a.y, b.y, a.x * b.x)); }

struct OrcParams {
  int kind;
  double particle_radius, h, sigma;
  double n_full, tot_min, lattice_grad;
  double wall_offset, wall_amplitude, taper0, taper1, reach;
  double tol_den, tol_div, max_error_factor;
  int min_it, max_it;
  double omega, warm_den, warm_div, min_nb;
  int divergence_solve, two_sided;
  double xsph_c;
  int capacity;
  double v_sep, relief_speed, project_eps;
  int has_bounds;
  double bounds_lo[3], bounds_hi[3];
  int cg;  // pressure iteration: 1 projected preconditioned CG (krylov.py), 0 relaxed Jacobi
  int wall_friction;  // Config.wall_friction: Coulomb friction of lone particles and projections on shape walls
  double jitter_speed;  // Config.rest_jitter_speed (0: the resting-jitter rule is off)
  double jitter_ratio;  // Config.rest_jitter_flow_ratio
  double tol_den_min;   // min(Config.min_density_error, max_density_error)
};

// Kernel constants in the working precision, derived from double host values exactly as the CUDA side does.
template <class R> struct KC {
  int kind;
  R h, inv_h, h2, sigma, sig_h2, m6sig_h, m20sig_h2, r_min;
  void init(int k, double hd, double sigma_d) {
    kind = k;
    h = R(hd);
    inv_h = R(1.0 / hd);
    h2 = h * h;
    sigma = R(sigma_d);
    sig_h2 = R(sigma_d / (hd * hd));
    m6sig_h = R(-6.0 * sigma_d / hd);
    m20sig_h2 = R(-20.0 * sigma_d / (hd * hd));
    r_min = R(1.0e-9 * hd);
  }
};

// W(r) and F(r) = (dW/dr)/r from r^2 (kernels.py:41-77); grad W_ij = (x_i - x_j) F.
template <class R> inline void wf(const KC<R>& k, R r2, R& W, R& F) {
  R r = std::sqrt(r2);
  R q = r * k.inv_h;
  if (q >= R(1)) { W = R(0); F = R(0); return; }
  if (k.kind == 0) {
    if (q <= R(0.5)) {
      W = k.sigma * fma_(R(6) * (q * q), q - R(1), R(1));
      F = k.sig_h2 * fma_(R(18), q, R(-12));
    } else {
      R s = R(1) - q;
      R s2 = s * s;
      W = k.sigma * (R(2) * (s2 * s));
      F = (k.m6sig_h * s2) / r;
    }
  } else {
    R s = R(1) - q;
    R s2 = s * s;
    W = k.sigma * ((s2 * s2) * fma_(R(4), q, R(1)));
    F = k.m20sig_h2 * (s2 * s);
  }
  if (r <= k.r_min) F = R(0);
}

// Psi(d) and dPsi/dd of a flat solid half-space at signed distance d (kernels.py:80-138, curvature H = 0).
// Cubic: p(y) = 1.4 - 8y^2 + 24y^4 - 19.2y^5 (y <= 1/2), (1-y)^4 (1.6 + 6.4y) (y > 1/2);
// G0(y) = int_0^y p = 1.4y - 8/3 y^3 + 4.8y^5 - 3.2y^6 (y <= 1/2), 1/2 - (1-y)^5 (1.6 - 16/15 (1-y)) (y > 1/2).
// Wendland C2: p(y) = 1.5 - 10.5y^2 + 52.5y^4 - 84y^5 + 52.5y^6 - 12y^7, G0 its integral.
template <class R> inline void halfspace(const KC<R>& k, R d, R& psi, R& dpsi) {
  if (d >= k.h) { psi = R(0); dpsi = R(0); return; }
  R z = clampr(-d * k.inv_h, R(-1), R(1));
  R y = std::fabs(z);
  R g0, p;
  if (k.kind == 0) {
    if (y <= R(0.5)) {
      R y2 = y * y;
      g0 = y * fma_(y2, fma_(y2, fma_(R(-3.2), y, R(4.8)), R(-2.66666666666666667)), R(1.4));
      p = fma_(y2, fma_(y2, fma_(R(-19.2), y, R(24)), R(-8)), R(1.4));
    } else {
      R u = R(1) - y;
      R u2 = u * u;
      R u4 = u2 * u2;
      g0 = R(0.5) - (u4 * u) * fma_(R(-1.06666666666666667), u, R(1.6));
      p = u4 * fma_(R(6.4), y, R(1.6));
    }
  } else {
    R y2 = y * y;
    g0 = y * fma_(y2, fma_(y2, fma_(y, fma_(y, fma_(R(-1.5), y, R(7.5)), R(-14)), R(10.5)), R(-3.5)), R(1.5));
    p = fma_(y2, fma_(y2, fma_(y, fma_(y, fma_(R(-12), y, R(52.5)), R(-84)), R(52.5)), R(-10.5)), R(1.5));
  }
  psi = (z < R(0)) ? R(0.5) - g0 : R(0.5) + g0;
  dpsi = (d > -k.h) ? -p * k.inv_h : R(0);
}

// The distance at which a flat wall covers c of the support (particle_walls.py:87-98).
template <class R> inline R colour_distance(const KC<R>& k, R c) {
  R lo = -k.h, hi = k.h;
  for (int it = 0; it < BISECT; ++it) {
    R mid = R(0.5) * (lo + hi);
    R psi, dpsi;
    halfspace(k, mid, psi, dpsi);
    if (psi > c) lo = mid; else hi = mid;
  }
  return R(0.5) * (lo + hi);
}

inline int64_t to_fixed(float m) { return (int64_t)std::llround((double)m * 1099511627776.0); }

template <class R> inline V3<R> quat_rotate(const float* qv, V3<R> v) {
  // v' = v (2w^2 - 1) + 2w (u x v) + 2u (u . v), u = (qx, qy, qz)
  R ux = R(qv[0]), uy = R(qv[1]), uz = R(qv[2]), w = R(qv[3]);
  R a = R(2) * (w * w) - R(1);
  R cx = uy * v.z - uz * v.y, cy = uz * v.x - ux * v.z, cz = ux * v.y - uy * v.x;
  R b = R(2) * w;
  R d = R(2) * ((ux * v.x + uy * v.y) + uz * v.z);
  return {(v.x * a + cx * b) + ux * d, (v.y * a + cy * b) + uy * d, (v.z * a + cz * b) + uz * d};
}

// --------------------------------------------------------------------------------------------- reductions
// Per-world float64 sum and max of a per-particle float array over contiguous world ranges, in this fixed order:
// chunks of 256 consecutive particles aligned to each world start; inside a chunk lane l holds v[b + l] (0 past the
// end), each group of 32 lanes folds with offsets 16, 8, 4, 2, 1 (lane l += lane l + off), then the 8 group sums
// fold with offsets 4, 2, 1. A world's 256 lanes then take chunks l, l + 256, ... serially and fold the same way.
inline double fold256(double* x) {
  for (int g = 0; g < 8; ++g) {
    double* y = x + 32 * g;
    for (int off = 16; off >= 1; off >>= 1)
      for (int l = 0; l < off; ++l) y[l] = y[l] + y[l + off];
  }
  double s[8];
  for (int g = 0; g < 8; ++g) s[g] = x[32 * g];
  for (int off = 4; off >= 1; off >>= 1)
    for (int l = 0; l < off; ++l) s[l] = s[l] + s[l + off];
  return s[0];
}

template <class R>
void world_sum(int W, const int* ws, const R* v, double* out, float* out_max) {
  const int CH = 256;
  for (int w = 0; w < W; ++w) {
    int lo = ws[w], hi = ws[w + 1];
    std::vector<double> part;
    float mx = -3.4e38f;
    for (int b = lo; b < hi; b += CH) {
      double x[256];
      for (int l = 0; l < CH; ++l) {
        int i = b + l;
        x[l] = (i < hi) ? (double)v[i] : 0.0;
        if (i < hi) mx = maxr(mx, (float)v[i]);
      }
      part.push_back(fold256(x));
    }
    double x[256];
    for (int l = 0; l < CH; ++l) {
      double a = 0.0;
      for (size_t c = l; c < part.size(); c += CH) a = a + part[c];
      x[l] = a;
    }
    out[w] = fold256(x);
    if (out_max) out_max[w] = maxr(mx, 0.0f);
  }
}

// ------------------------------------------------------------------------------------------------ solver
struct Emitter {
  int world;
  float xform[7];
  float vel[3];
  float interval;
  std::vector<float> offsets;  // n_layer x 3
  std::vector<int> pool;
  int enabled = 1;
  float t_acc = 0.0f;
  int cursor = 0;
};
struct Sink {
  int world;
  float xform[7];
  float half[3];
};

template <class R> struct Solver {
  OrcParams P;
  KC<R> kc;
  int n = 0, W = 0, K = 64;
  std::vector<int> ws;
  std::vector<float> mass, rho0, wall_vol, gravity;
  std::vector<int> flags, world;
  std::vector<int8_t> phase;
  std::vector<V3<R>> q, v, vtmp, acc;
  std::vector<R> kv, kd;
  // per step
  std::vector<int> group, cnt, nbr;
  // boundary slots, [i * NS + k]: shape id (-1 empty; S = the particle wall), Psi, phi, grad Psi, wall velocity, and
  // the start-of-step plane (closest point, outward normal; world frame for the particle wall, shape frame for a box)
  std::vector<int> s_cnt, s_shape;
  std::vector<R> s_psi, s_phi;
  std::vector<V3<R>> s_g, s_vb, s_xbl, s_nbl;
  // the liquid's static axis-aligned box walls (layout.py:207-246): per-world CSR of shape ids, centre, half extents,
  // bounding radius and friction
  int S = 0;
  std::vector<int> sh_start, sh_ids;
  std::vector<float> sh_pos, sh_half, sh_radius, sh_mu;
  std::vector<int> sh_geo;  // newton GeoType per shape (box, sphere, capsule and cylinder along z, plane facing +z)
  std::vector<float> sh_quat;  // [S][4] the shape frame's rotation (x, y, z, w)
  double sweep_len = 1.0e30;
  std::vector<int> swept;
  std::vector<R> ratio, alpha, neff, active, reg, src, kappa, lower, err;
  // per world
  std::vector<int> overflow, escaped, projected, nonfinite, emit_overflow;
  std::vector<int> iters_den, iters_div, converged, iters;
  std::vector<float> den_err, div_err, den_err_max, max_speed, err_mean, den_tol;
  // the resting-jitter rule (solve_driver.py): per-world flow sums of the step's start state (sum v_z, count,
  // sum v_x, sum v_y) and the density solve's tolerance factor
  std::vector<double> flow_sum[4];
  std::vector<float> tol_scale;
  std::vector<int64_t> mass_in, mass_out, mass0;
  std::vector<double> n_active;
  std::vector<Emitter> emitters;
  std::vector<Sink> sinks;
  int nthreads = 1;

  bool is_fluid(int i) const { return (flags[i] & FLAG_ACTIVE) != 0 && phase[i] >= 1; }

  void init() {
    K = P.capacity;
    kc.init(P.kind, P.h, P.sigma);
    auto zr = [&](std::vector<R>& a) { a.assign(n, R(0)); };
    auto z3 = [&](std::vector<V3<R>>& a) { a.assign(n, V3<R>{R(0), R(0), R(0)}); };
    z3(q); z3(v); z3(vtmp); z3(acc);
    zr(kv); zr(kd);
    group.assign(n, -1); cnt.assign(n, 0); nbr.assign((size_t)n * K, -1);
    s_cnt.assign(n, 0);
    s_shape.assign((size_t)n * NS, -1);
    s_psi.assign((size_t)n * NS, R(0)); s_phi.assign((size_t)n * NS, R(0));
    const V3<R> z0{R(0), R(0), R(0)};
    s_g.assign((size_t)n * NS, z0); s_vb.assign((size_t)n * NS, z0); s_xbl.assign((size_t)n * NS, z0);
    s_nbl.assign((size_t)n * NS, z0);
    sweep_len = 0.5 * P.h;
    sh_start.assign(W + 1, 0);
    zr(ratio); zr(alpha); zr(neff); zr(active); zr(reg); zr(src); zr(kappa); zr(lower); zr(err);
    auto zi = [&](std::vector<int>& a) { a.assign(W, 0); };
    zi(overflow); zi(escaped); zi(projected); zi(nonfinite); zi(emit_overflow); zi(swept);
    zi(iters_den); zi(iters_div); zi(converged); zi(iters);
    auto zf = [&](std::vector<float>& a) { a.assign(W, 0.0f); };
    zf(den_err); zf(div_err); zf(den_err_max); zf(max_speed); zf(err_mean); zf(den_tol);
    mass_in.assign(W, 0); mass_out.assign(W, 0); mass0.assign(W, 0);
    n_active.assign(W, 0.0);
  }

  void init_mass() {
    for (int w = 0; w < W; ++w) mass0[w] = 0;
    for (int i = 0; i < n; ++i)
      if (is_fluid(i)) mass0[world[i]] += to_fixed(mass[i]);
  }

  // ------------------------------------------------------------------- grid (this oracle's own, per world)
  struct Grid {
    double lo[3];
    int dim[3];
    double cw;
    std::vector<int> start, ids;  // counting sort of members by cell
    int cell_of(const V3<R>& x, int* c) const {
      double p[3] = {(double)x.x, (double)x.y, (double)x.z};
      for (int a = 0; a < 3; ++a) {
        double f = std::floor((p[a] - lo[a]) / cw);
        int ci = (f < 0.0) ? 0 : (f > dim[a] - 1 ? dim[a] - 1 : (int)f);
        if (!(f == f)) ci = 0;
        c[a] = ci;
      }
      return (c[2] * dim[1] + c[1]) * dim[0] + c[0];
    }
  };
  std::vector<Grid> fluid_grid, wall_grid;

  void build_grid(Grid& g, const std::vector<int>& members, const double* lo, const int* dim, double cw) {
    for (int a = 0; a < 3; ++a) { g.lo[a] = lo[a]; g.dim[a] = dim[a]; }
    g.cw = cw;
    size_t nc = (size_t)dim[0] * dim[1] * dim[2];
    g.start.assign(nc + 1, 0);
    std::vector<int> key(members.size());
    for (size_t m = 0; m < members.size(); ++m) {
      int c[3];
      key[m] = g.cell_of(q[members[m]], c);
      g.start[key[m] + 1]++;
    }
    for (size_t c = 0; c < nc; ++c) g.start[c + 1] += g.start[c];
    g.ids.assign(members.size(), 0);
    std::vector<int> cur(g.start.begin(), g.start.end() - 1);
    for (size_t m = 0; m < members.size(); ++m) g.ids[cur[key[m]]++] = members[m];
  }

  void build_groups_and_grids() {
    for (int i = 0; i < n; ++i) {
      int g = -1;
      if ((flags[i] & FLAG_ACTIVE) != 0 && phase[i] >= 1) g = world[i];
      else if (wall_vol[i] > 0.0f && (flags[i] & FLAG_ACTIVE) != 0 && world[i] >= 0) g = -2 - world[i];
      group[i] = g;
    }
    fluid_grid.assign(W, Grid());
    wall_grid.assign(W, Grid());
    const double cw = 1.01 * P.h;
    for (int w = 0; w < W; ++w) {
      std::vector<int> fl, wl;
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      for (int i = ws[w]; i < ws[w + 1]; ++i) {
        if (group[i] == w) fl.push_back(i);
        else if (group[i] == -2 - w) wl.push_back(i);
        else continue;
        double p[3] = {(double)q[i].x, (double)q[i].y, (double)q[i].z};
        for (int a = 0; a < 3; ++a)
          if (std::isfinite(p[a])) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
      }
      int dim[3];
      double cww = cw;
      for (;;) {  // cells never narrower than h; coarser where a world's box is huge (escaped particles)
        double cells = 1.0;
        for (int a = 0; a < 3; ++a) {
          if (!(lo[a] <= hi[a])) { lo[a] = 0.0; hi[a] = 0.0; }
          dim[a] = (int)std::floor((hi[a] - lo[a]) / cww) + 1;
          cells *= dim[a];
        }
        if (cells <= 6.4e7) break;
        cww *= 2.0;
      }
      build_grid(fluid_grid[w], fl, lo, dim, cww);
      build_grid(wall_grid[w], wl, lo, dim, cww);
    }
  }

  template <class Fn> void for_each_near(const Grid& g, const V3<R>& x, Fn fn) const {
    int c[3];
    g.cell_of(x, c);
    for (int dz = -1; dz <= 1; ++dz) {
      int z = c[2] + dz;
      if (z < 0 || z >= g.dim[2]) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        int y = c[1] + dy;
        if (y < 0 || y >= g.dim[1]) continue;
        for (int dx = -1; dx <= 1; ++dx) {
          int xx = c[0] + dx;
          if (xx < 0 || xx >= g.dim[0]) continue;
          int cell = (z * g.dim[1] + y) * g.dim[0] + xx;
          for (int m = g.start[cell]; m < g.start[cell + 1]; ++m) fn(g.ids[m]);
        }
      }
    }
  }

  // neighbors.py:160-195: ascending ids j != i of the same group with |x_j - x_i|^2 < h^2, lowest K kept
  void build_lists() {
    std::vector<int> ovf(W, 0);
#pragma omp parallel num_threads(nthreads)
    {
      std::vector<int> cand;
      std::vector<int> ovf_local(W, 0);
#pragma omp for schedule(dynamic, 256)
      for (int i = 0; i < n; ++i) {
        int g = group[i];
        if (g < 0) { cnt[i] = 0; continue; }
        cand.clear();
        const V3<R> xi = q[i];
        for_each_near(fluid_grid[g], xi, [&](int j) {
          if (j == i) return;
          V3<R> d = sub(q[j], xi);
          if (dot_plain(d, d) < kc.h2) cand.push_back(j);
        });
        std::sort(cand.begin(), cand.end());
        int total = (int)cand.size();
        int m = std::min(total, K);
        for (int k = 0; k < m; ++k) nbr[(size_t)i * K + k] = cand[k];
        cnt[i] = m;
        if (total > K) ovf_local[g]++;
      }
#pragma omp critical
      for (int w = 0; w < W; ++w) ovf[w] += ovf_local[w];
    }
    for (int w = 0; w < W; ++w) overflow[w] += ovf[w];
  }

  // newton geometry/kernels.py:310-370 (sdf_box, sdf_box_grad): signed distance of the axis-aligned box of half
  // extents hx at shape-local p, and its outward unit gradient
  static R box_sdf(const V3<R>& p, const float* hx) {
    R qx = std::fabs(p.x) - R(hx[0]), qy = std::fabs(p.y) - R(hx[1]), qz = std::fabs(p.z) - R(hx[2]);
    V3<R> e{maxr(qx, R(0)), maxr(qy, R(0)), maxr(qz, R(0))};
    return std::sqrt(dot_plain(e, e)) + minr(maxr(qx, maxr(qy, qz)), R(0));
  }
  static V3<R> normalized(const V3<R>& a) {
    R l = std::sqrt(dot_plain(a, a));
    if (l > R(0)) return {a.x / l, a.y / l, a.z / l};
    return {R(0), R(0), R(0)};
  }
  static V3<R> box_grad(const V3<R>& p, const float* hx) {
    const R h0 = R(hx[0]), h1 = R(hx[1]), h2 = R(hx[2]);
    R qx = std::fabs(p.x) - h0, qy = std::fabs(p.y) - h1, qz = std::fabs(p.z) - h2;
    if (qx > R(0) || qy > R(0) || qz > R(0)) {
      V3<R> c{clampr(p.x, -h0, h0), clampr(p.y, -h1, h1), clampr(p.z, -h2, h2)};
      return normalized(sub(p, c));
    }
    R sx = p.x < R(0) ? R(-1) : R(1), sy = p.y < R(0) ? R(-1) : R(1), sz = p.z < R(0) ? R(-1) : R(1);
    if ((qx > qy && qx > qz) || (qy == R(0) && qz == R(0))) return {sx, R(0), R(0)};
    if ((qy > qx && qy > qz) || (qx == R(0) && qz == R(0))) return {R(0), sy, R(0)};
    return {R(0), R(0), sz};
  }
  // newton eval_shape_sdf (soft_contacts_sdf.py:249-280) for the analytic shapes of this path: the signed distance of
  // shape sh at shape-local p (box sdf_box; sphere sdf_sphere; capsule along z sdf_capsule; plane facing +z
  // _eval_plane_sdf) and its outward unit gradient (sdf_*_grad; +z at a sphere's centre or a capsule's
  // axis, -z below its lower cap; +z for a plane)
  static constexpr int GEO_PLANE = 1, GEO_SPHERE = 3, GEO_CAPSULE = 4, GEO_CYLINDER = 6, GEO_BOX = 7;
  // the shape's frame: identity rotations leave vectors as they are (an unrotated frame is a translation only)
  bool rotated(int sh) const {
    const float* q = &sh_quat[4 * sh];
    return !(q[0] == 0.0f && q[1] == 0.0f && q[2] == 0.0f && q[3] == 1.0f);
  }
  V3<R> to_frame(int sh, const V3<R>& v) const {
    if (!rotated(sh)) return v;
    const float* q = &sh_quat[4 * sh];
    const float c[4] = {-q[0], -q[1], -q[2], q[3]};
    return quat_rotate(c, v);
  }
  V3<R> from_frame(int sh, const V3<R>& v) const { return rotated(sh) ? quat_rotate(&sh_quat[4 * sh], v) : v; }
  // geometry/kernels.py:515-600 (sdf_cylinder, sdf_cylinder_grad; straight sides along z)
  R cylinder_phi(const float* s, const V3<R>& p) const {
    const V3<R> v{p.x, p.y, R(0)};
    const R rho = std::sqrt(dot_plain(v, v)), dx = rho - R(s[0]), dy = std::fabs(p.z) - R(s[1]);
    const R ex = maxr(dx, R(0)), ey = maxr(dy, R(0));
    return minr(maxr(dx, dy), R(0)) + std::sqrt(ex * ex + ey * ey);
  }
  V3<R> cylinder_grad(const float* s, const V3<R>& p) const {
    const V3<R> v{p.x, p.y, R(0)};
    const R rho = std::sqrt(dot_plain(v, v)), dx = rho - R(s[0]), dy = std::fabs(p.z) - R(s[1]);
    V3<R> rad{R(0), R(0), R(1)};
    if (rho > R(1.0e-8)) rad = {p.x / rho, p.y / rho, R(0)};
    const R az = p.z < R(0) ? R(-1) : R(1);
    if (dx > R(0) && dy > R(0)) {
      const V3<R> g{rad.x * dx, rad.y * dx, fma_(az, dy, rad.z * dx)};
      const R gl = std::sqrt(dot_plain(g, g));
      if (gl > R(1.0e-8)) return {g.x / gl, g.y / gl, g.z / gl};
      return rad;
    }
    if (dx > dy) return rad;
    return {R(0), R(0), az};
  }
  // soft_contacts_sdf.py:73-102 (_eval_plane_sdf, depth 0): infinite unless width and length are both positive; a
  // finite plane is a two-sided sheet, its z over the footprint from above, else the distance to its nearest point
  static bool plane_over(const float* s, const V3<R>& p) {
    const R hw = R(0.5) * R(s[0]), hl = R(0.5) * R(s[1]);
    return !(hw > R(0) && hl > R(0)) || (std::fabs(p.x) <= hw && std::fabs(p.y) <= hl && p.z >= R(0));
  }
  static V3<R> plane_delta(const float* s, const V3<R>& p) {
    const R hw = R(0.5) * R(s[0]), hl = R(0.5) * R(s[1]);
    return {p.x - clampr(p.x, -hw, hw), p.y - clampr(p.y, -hl, hl), p.z - R(0)};
  }
  R shape_phi(int sh, const V3<R>& p) const {
    const float* s = &sh_half[3 * sh];
    const int g = sh_geo[sh];
    if (g == GEO_BOX) return box_sdf(p, s);
    if (g == GEO_CYLINDER) return cylinder_phi(s, p);
    if (g == GEO_PLANE) {
      if (plane_over(s, p)) return p.z;
      const V3<R> d = plane_delta(s, p);
      return std::sqrt(dot_plain(d, d));
    }
    R cz = p.z;
    if (g == GEO_CAPSULE) cz = p.z > R(s[1]) ? p.z - R(s[1]) : (p.z < -R(s[1]) ? p.z + R(s[1]) : R(0));
    const V3<R> v{p.x, p.y, cz};
    return std::sqrt(dot_plain(v, v)) - R(s[0]);
  }
  V3<R> shape_grad(int sh, const V3<R>& p) const {
    const float* s = &sh_half[3 * sh];
    const int g = sh_geo[sh];
    if (g == GEO_BOX) return box_grad(p, s);
    if (g == GEO_CYLINDER) return cylinder_grad(s, p);
    if (g == GEO_PLANE) {
      if (plane_over(s, p)) return {R(0), R(0), R(1)};
      const V3<R> d = plane_delta(s, p);
      const R l = std::sqrt(dot_plain(d, d));
      if (l > R(0)) return {d.x / l, d.y / l, d.z / l};
      return {R(0), R(0), R(1)};
    }
    R cz = p.z, dz = R(1);
    if (g == GEO_CAPSULE) {
      if (p.z > R(s[1])) cz = p.z - R(s[1]);
      else if (p.z < -R(s[1])) { cz = p.z + R(s[1]); dz = R(-1); }
      else cz = R(0);
    }
    const V3<R> v{p.x, p.y, cz};
    const R l = std::sqrt(dot_plain(v, v));
    if (l > R(1.0e-8)) return {v.x / l, v.y / l, v.z / l};
    return {R(0), R(0), dz};
  }
  V3<R> shape_local(int sh, const V3<R>& x) const {  // static shape: its frame's origin and rotation
    return to_frame(sh, {x.x - R(sh_pos[3 * sh]), x.y - R(sh_pos[3 * sh + 1]), x.z - R(sh_pos[3 * sh + 2])});
  }
  V3<R> shape_world(int sh, const V3<R>& l) const {  // a world-oriented offset from the shape's origin to the point
    return {l.x + R(sh_pos[3 * sh]), l.y + R(sh_pos[3 * sh + 1]), l.z + R(sh_pos[3 * sh + 2])};
  }

  // boundary_slots.py:13-37: (sh, phi) into particle i's phi-ascending row of n_ slots; the slot used, or -1
  int slot_insert(int i, int n_, int sh, R phi) {
    int* shp = &s_shape[(size_t)i * NS];
    R* ph = &s_phi[(size_t)i * NS];
    int pos = n_, k = n_ - 1;
    while (k >= 0) {
      if (ph[k] <= phi) break;
      pos = k;
      --k;
    }
    if (pos >= NS) return -1;
    for (k = n_ >= NS ? NS - 1 : n_; k > pos; --k) {
      shp[k] = shp[k - 1];
      ph[k] = ph[k - 1];
    }
    shp[pos] = sh;
    ph[pos] = phi;
    return pos;
  }

  // boundary_slots.py:59-102: a wall (sh, phi, world normal nrm) into the row; a full row drops the farthest
  // same-facing duplicate (cos > COS_SAME) of its four slots and the new wall, never one nearer than `near`, with
  // none the farthest of the five. nr holds the slots' normals. 1 if the wall was kept.
  int shape_insert(int i, int n_, int sh, R phi, const V3<R>& nrm, V3<R>* nr, R near) {
    if (n_ < NS) {
      const int r = slot_insert(i, n_, sh, phi);
      if (r < 0) return 0;
      for (int k = n_; k > r; --k) nr[k] = nr[k - 1];
      nr[r] = nrm;
      return 1;
    }
    int* shp = &s_shape[(size_t)i * NS];
    R* ph = &s_phi[(size_t)i * NS];
    const R cs = R(COS_SAME);
    int ev = -1;
    R ev_phi = R(-1);
    for (int m = 0; m < NS; ++m)
      if (phi >= near && ph[m] <= phi && dot_plain(nr[m], nrm) > cs) { ev = 4; ev_phi = phi; }
    for (int k = 0; k < NS; ++k) {
      const R pk = ph[k];
      int dup = 0;
      for (int m = 0; m < NS; ++m)
        if (m != k && ph[m] <= pk && dot_plain(nr[m], nr[k]) > cs) dup = 1;
      if (phi <= pk && dot_plain(nrm, nr[k]) > cs) dup = 1;
      if (dup == 1 && pk >= near && pk > ev_phi) { ev = k; ev_phi = pk; }
    }
    if (ev < 0 && phi < ph[3]) ev = 3;
    if (ev < 0 || ev == 4) return 0;
    for (int k = ev; k < NS - 1; ++k) { shp[k] = shp[k + 1]; ph[k] = ph[k + 1]; nr[k] = nr[k + 1]; }
    int pos = NS - 1;
    while (pos > 0 && ph[pos - 1] > phi) { shp[pos] = shp[pos - 1]; ph[pos] = ph[pos - 1]; nr[pos] = nr[pos - 1]; --pos; }
    shp[pos] = sh;
    ph[pos] = phi;
    nr[pos] = nrm;
    return 1;
  }

  // (Psi, dPsi) of a wall at distance phi: A Psi(phi + delta) with the C1 taper (boundary.py:241-251, kernels.py)
  void wall_volume(R phi, R& psi, R& dpsi) const {
    const R offset = R(P.wall_offset), amp = R(P.wall_amplitude), t0 = R(P.taper0), t1 = R(P.taper1);
    halfspace(kc, phi + offset, psi, dpsi);
    psi = psi * amp;
    dpsi = dpsi * amp;
    if (phi > t0) {  // C1 taper between the first and second lattice layer
      R L = t1 - t0;
      R t = minr((phi - t0) / L, R(1));
      R sm = R(1) - (t * t) * (R(3) - R(2) * t);
      R dsm = ((R(6) * t) * (t - R(1))) / L;
      R p0 = psi;
      psi = p0 * sm;
      dpsi = fma_(p0, dsm, dpsi * sm);
    }
  }

  // boundary.py:190-238 (find), 254-396 (fill, combine) with particle_walls.py:65-119: fluid particle i's slots
  void wall_slots() {
    const R reach = R(P.reach), offset = R(P.wall_offset), near = R(0.1) * kc.h;
#pragma omp parallel num_threads(nthreads)
    {
      struct C { int j; R wj, F; V3<R> d; };
      std::vector<C> cand;
#pragma omp for schedule(dynamic, 256)
      for (int i = 0; i < n; ++i) {
        s_cnt[i] = 0;
        for (int k = 0; k < NS; ++k) {
          s_shape[(size_t)i * NS + k] = -1;
          s_psi[(size_t)i * NS + k] = R(0);
          s_g[(size_t)i * NS + k] = {R(0), R(0), R(0)};
        }
        if (!is_fluid(i)) continue;
        const int w = world[i];
        const V3<R> x = q[i];
        int ns = 0;
        V3<R> nr[NS];
        // the world's box walls within the reach (boundary.py:211-222)
        for (int c = sh_start[w]; c < sh_start[w + 1]; ++c) {
          const int sh = sh_ids[c];
          const V3<R> d{x.x - R(sh_pos[3 * sh]), x.y - R(sh_pos[3 * sh + 1]), x.z - R(sh_pos[3 * sh + 2])};
          if (sh_geo[sh] != GEO_PLANE && std::sqrt(dot_plain(d, d)) > R(sh_radius[sh]) + kc.h) continue;
          const V3<R> xl = shape_local(sh, x);
          const R phi = shape_phi(sh, xl);
          if (phi < reach && phi + offset < kc.h) {
            const V3<R> nw = from_frame(sh, normalized(shape_grad(sh, xl)));
            if (shape_insert(i, ns, sh, phi, nw, nr, near) > 0 && ns < NS) ++ns;
          }
        }
        // the particle wall: colour sums in ascending wall-particle id (particle_walls.py:65-107)
        cand.clear();
        for_each_near(wall_grid[w], x, [&](int j) {
          V3<R> d = sub(x, q[j]);
          R Wv, F;
          wf(kc, dot_plain(d, d), Wv, F);
          R wj = R(wall_vol[j]) * Wv;
          if (wj > R(0)) cand.push_back({j, wj, F, d});
        });
        R pw_phi = R(0);
        V3<R> pw_n{R(0), R(0), R(0)}, pw_v{R(0), R(0), R(0)};
        bool pw = false;
        if (!cand.empty()) {
          std::sort(cand.begin(), cand.end(), [](const C& a, const C& b) { return a.j < b.j; });
          R c = R(0);
          V3<R> gc{R(0), R(0), R(0)}, mv{R(0), R(0), R(0)};
          for (const C& e : cand) {
            R vol = R(wall_vol[e.j]);
            c = c + e.wj;
            gc.x = fma_(vol, e.d.x * e.F, gc.x);
            gc.y = fma_(vol, e.d.y * e.F, gc.y);
            gc.z = fma_(vol, e.d.z * e.F, gc.z);
            mv.x = fma_(e.wj, v[e.j].x, mv.x);
            mv.y = fma_(e.wj, v[e.j].y, mv.y);
            mv.z = fma_(e.wj, v[e.j].z, mv.z);
          }
          mv = {mv.x / c, mv.y / c, mv.z / c};
          R lg = std::sqrt(dot_plain(gc, gc));
          if (!(c < R(C_MIN) || lg <= R(0))) {
            R phi = colour_distance(kc, minr(c, R(1)));
            if (phi < reach && phi + offset < kc.h) {
              if (slot_insert(i, ns, S, phi) >= 0 && ns < NS) ++ns;
              pw = true;
              pw_phi = phi;
              pw_n = {-gc.x / lg, -gc.y / lg, -gc.z / lg};
              pw_v = mv;
            }
          }
        }
        (void)pw;
        s_cnt[i] = ns;
        // fill (boundary.py:254-334): a box's slot from its SDF, the particle wall's from its plane
        for (int k = 0; k < ns; ++k) {
          const size_t o = (size_t)i * NS + k;
          const int sh = s_shape[o];
          R phi, psi, dpsi;
          V3<R> nrm;
          if (sh == S) {
            phi = pw_phi;
            nrm = pw_n;
            s_vb[o] = pw_v;
            s_xbl[o] = {fma_(-phi, nrm.x, x.x), fma_(-phi, nrm.y, x.y), fma_(-phi, nrm.z, x.z)};
            s_nbl[o] = nrm;
          } else {
            const V3<R> xl = shape_local(sh, x);
            phi = shape_phi(sh, xl);
            const V3<R> gl = shape_grad(sh, xl);
            nrm = normalized(gl);
            s_xbl[o] = from_frame(sh, V3<R>{fma_(-phi, nrm.x, xl.x), fma_(-phi, nrm.y, xl.y), fma_(-phi, nrm.z, xl.z)});
            nrm = from_frame(sh, nrm);  // slots hold world normals and world-oriented closest points
            s_nbl[o] = nrm;
            s_vb[o] = {R(0), R(0), R(0)};
          }
          wall_volume(phi, psi, dpsi);
          s_phi[o] = phi;
          s_psi[o] = psi;
          s_g[o] = {dpsi * nrm.x, dpsi * nrm.y, dpsi * nrm.z};
        }
        // boundary.py:354-396: overlapping walls by inclusion-exclusion (psi as filled, gradients as they are
        // rewritten slot by slot)
        if (ns > 1) {
          R ps[NS];
          for (int k = 0; k < NS; ++k) ps[k] = s_psi[(size_t)i * NS + k];
          for (int b = 0; b < ns; ++b) {
            const size_t ob_i = (size_t)i * NS + b;
            const V3<R> gb = s_g[ob_i];
            R ob = R(0), sb = R(0);
            for (int c = 0; c < ns; ++c) {
              if (c == b) continue;
              const V3<R> gcv = s_g[(size_t)i * NS + c];
              const R lb = std::sqrt(dot_plain(gb, gb)), lc = std::sqrt(dot_plain(gcv, gcv));
              R cbc = R(0);
              if (lb > R(0) && lc > R(0)) cbc = clampr(dot_plain(gb, gcv) / (lb * lc), R(-1), R(1));
              ob = ob + (R(1) - std::fabs(cbc)) * ps[c];
              if (cbc > R(0) && (ps[c] > ps[b] || (ps[c] == ps[b] && c < b))) sb = sb + cbc;
            }
            ob = minr(ob, R(1));
            s_psi[ob_i] = ps[b] * maxr((R(1) - R(0.5) * ob) - sb, R(0));
            const R f = maxr((R(1) - ob) - sb, R(0));
            s_g[ob_i] = {gb.x * f, gb.y * f, gb.z * f};
          }
        }
      }
    }
  }

  // pressure.py:144-193
  void density_alpha() {
    const R n_full = R(P.n_full), tot_min = R(P.tot_min);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) { ratio[i] = alpha[i] = neff[i] = active[i] = reg[i] = R(0); continue; }
      const V3<R> xi = q[i];
      R mi = R(mass[i]);
      R inv_r0 = R(1) / R(rho0[i]);
      R bi = mi * inv_r0;
      R rho = mi * kc.sigma;
      V3<R> G{R(0), R(0), R(0)};
      R sq = R(0);
      const int* row = &nbr[(size_t)i * K];
      for (int k = 0; k < cnt[i]; ++k) {
        int j = row[k];
        V3<R> rv = sub(xi, q[j]);
        R r2 = dot_plain(rv, rv);
        R Wv, F;
        wf(kc, r2, Wv, F);
        R mj = R(mass[j]);
        rho = fma_(mj, Wv, rho);
        R a = mj * inv_r0;
        R aF = a * F;
        G.x = fma_(aF, rv.x, G.x);
        G.y = fma_(aF, rv.y, G.y);
        G.z = fma_(aF, rv.z, G.z);
        sq = fma_(bi * a, (F * F) * r2, sq);
      }
      R psi = R(0), lam = R(0);  // boundary slots, nearest first; lam: the opposing-wall compliance
      for (int b = 0; b < s_cnt[i]; ++b) {
        const size_t o = (size_t)i * NS + b;
        psi = psi + s_psi[o];
        G.x = G.x + s_g[o].x;
        G.y = G.y + s_g[o].y;
        G.z = G.z + s_g[o].z;
        for (int c = b + 1; c < s_cnt[i]; ++c)
          lam = lam + maxr(R(-2) * dot_plain(s_g[o], s_g[(size_t)i * NS + c]), R(0));
      }
      R tot = (dotf(G, G) + sq) + lam;
      lam = lam + maxr(tot_min - tot, R(0));
      tot = maxr(tot, tot_min);
      reg[i] = lam;
      ratio[i] = fma_(rho, inv_r0, psi);
      alpha[i] = (tot > R(1.0e-12)) ? R(1) / tot : R(0);
      neff[i] = fma_(psi, n_full, R(cnt[i]));
      active[i] = R(1);
    }
  }

  // pressure.py:196-261 (the lone-particle and two-sided branches included)
  void solve_init(bool div, R dt, R relief) {
    const R warm = R(div ? P.warm_div : P.warm_den), warm_den = R(P.warm_den), min_nb = R(P.min_nb);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) { src[i] = kappa[i] = lower[i] = R(0); continue; }
      const V3<R> xi = q[i], vi = v[i];
      R inv_r0 = R(1) / R(rho0[i]);
      R rate = R(0);
      const int* row = &nbr[(size_t)i * K];
      for (int k = 0; k < cnt[i]; ++k) {
        int j = row[k];
        V3<R> rv = sub(xi, q[j]);
        R Wv, F;
        wf(kc, dot_plain(rv, rv), Wv, F);
        R aF = (R(mass[j]) * inv_r0) * F;
        rate = fma_(aF, dotf(sub(vi, v[j]), rv), rate);
      }
      for (int b = 0; b < s_cnt[i]; ++b) {
        const size_t o = (size_t)i * NS + b;
        rate = rate + dotf(sub(vi, s_vb[o]), s_g[o]);
      }
      if (div) {
        R kdv = R(0);
        if (P.two_sided) kdv = maxr((warm_den * minr(kd[i], R(2.5e-4))) / (dt * dt), R(0));
        R lb = -kdv;
        R r = rate;
        if (kdv <= R(0)) { r = maxr(rate, R(0)); lb = R(0); }
        if (neff[i] < min_nb) { r = R(0); lb = R(0); }
        src[i] = r;
        lower[i] = lb;
        kappa[i] = maxr((warm * minr(kv[i], R(0.5))) / dt, lb);
      } else {
        R rs = fma_(dt, rate, ratio[i]);
        if (ratio[i] - R(1) > relief) rs = fma_(dt, rate, R(1) + relief);
        src[i] = rs;
        lower[i] = R(0);
        kappa[i] = (warm * minr(kd[i], R(2.5e-4))) / (dt * dt);
      }
    }
  }

  // pressure.py:264-277: a_i = -sum_j m_j (k_i/rho0_i + k_j/rho0_j) grad W_ij - k_i sum_b dPsi_b
  V3<R> pressure_accel(int i, const std::vector<R>& kr) const { return pressure_accel(i, kr, kappa); }

  // a_i of the pressure field whose kappa / rho0 is kr and whose kappa is kvec (slot term)
  V3<R> pressure_accel(int i, const std::vector<R>& kr, const std::vector<R>& kvec) const {
    const V3<R> xi = q[i];
    R ki = kr[i];
    V3<R> a{R(0), R(0), R(0)};
    const int* row = &nbr[(size_t)i * K];
    for (int k = 0; k < cnt[i]; ++k) {
      int j = row[k];
      V3<R> rv = sub(xi, q[j]);
      R Wv, F;
      wf(kc, dot_plain(rv, rv), Wv, F);
      R cF = (R(mass[j]) * (ki + kr[j])) * F;
      a.x = fma_(-cF, rv.x, a.x);
      a.y = fma_(-cF, rv.y, a.y);
      a.z = fma_(-cF, rv.z, a.z);
    }
    for (int b = 0; b < s_cnt[i]; ++b) {
      const R k = kvec[i];
      const V3<R> g = s_g[(size_t)i * NS + b];
      a.x = fma_(-k, g.x, a.x);
      a.y = fma_(-k, g.y, a.y);
      a.z = fma_(-k, g.z, a.z);
    }
    return a;
  }

  std::vector<R> kr;  // kappa / rho0, refreshed whenever kappa changes

  void refresh_kr() {
    kr.resize(n);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) kr[i] = kappa[i] / R(rho0[i]);
  }

  // pressure.py:280-291
  void accel_pass() {
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) { acc[i] = {R(0), R(0), R(0)}; continue; }
      if (converged[world[i]]) continue;
      acc[i] = pressure_accel(i, kr);
    }
  }

  // pressure.py:294-310: Ar_i of the accelerations in acc (the matrix-free product, before the compliance term)
  R accel_divergence(int i) const {
    const V3<R> xi = q[i], ai = acc[i];
    R inv_r0 = R(1) / R(rho0[i]);
    R ar = R(0);
    const int* row = &nbr[(size_t)i * K];
    for (int k = 0; k < cnt[i]; ++k) {
      int j = row[k];
      V3<R> rv = sub(xi, q[j]);
      R Wv, F;
      wf(kc, dot_plain(rv, rv), Wv, F);
      R aF = (R(mass[j]) * inv_r0) * F;
      ar = fma_(aF, dotf(sub(ai, acc[j]), rv), ar);
    }
    for (int b = 0; b < s_cnt[i]; ++b) ar = ar + dotf(ai, s_g[(size_t)i * NS + b]);
    return ar;
  }

  // pressure.py:294-352
  void jacobi_pass(bool div, R dt) {
    const R omega = R(P.omega), min_nb = R(P.min_nb);
    const R scale = div ? R(1) / dt : R(1) / (dt * dt);
    const R dtn = div ? dt : dt * dt;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) { err[i] = R(0); continue; }
      if (converged[world[i]]) continue;
      R ar = accel_divergence(i);
      ar = fma_(-reg[i], kappa[i], ar);
      ar = ar * dtn;
      R s = div ? -src[i] : R(1) - src[i];
      R r = s - ar;
      R lb = lower[i];
      R knew = maxr(kappa[i] - ((omega * r) * alpha[i]) * scale, lb);
      kappa[i] = knew;
      kr[i] = knew / R(rho0[i]);
      R e = maxr(-r, R(0));
      if (knew > lb) e = std::fabs(r);
      if (div) {
        if (neff[i] < min_nb) e = R(0);
        e = e * dt;
      }
      err[i] = e;
    }
  }

  // ---------------------------------------------------------------- projected preconditioned CG (krylov.py)
  // One CG per world on the bound-constrained DFSPH system w = A k - b, k >= k_lo (krylov.py:1-17). Operations
  // follow krylov.py:77-318 kernel by kernel; a + b c updates are fused (fma), dot products are the per-world
  // float64 sums of world_sum in particle order.
  std::vector<R> cg_pd, cg_pdr, cg_z, cg_w, cg_ap, cg_corr, cg_corrr, pair_x, pair_y;
  std::vector<int> cg_act, cg_restart;
  std::vector<double> cg_rz, cg_step, sum_x, sum_y;
  std::vector<float> cg_emax;

  bool cg_skip(int i, bool gated) const {
    const int w = world[i];
    return converged[w] != 0 || (gated && cg_restart[w] == 0);
  }

  // krylov.py:71-80: acc = pressure acceleration of the field vec (vr = vec / rho0)
  void cg_accel(const std::vector<R>& vec, const std::vector<R>& vr, bool gated) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) { acc[i] = {R(0), R(0), R(0)}; continue; }
      if (cg_skip(i, gated)) continue;
      acc[i] = pressure_accel(i, vr, vec);
    }
  }

  // krylov.py:83-101: out (+)= A vec (- b); pair.x = vec_i (A vec)_i
  void cg_apply(bool div, R dt, const std::vector<R>& vec, std::vector<R>& out, bool gated, bool bias,
                bool accumulate) {
    const R scale = div ? dt : dt * dt;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) { out[i] = R(0); pair_x[i] = R(0); pair_y[i] = R(0); continue; }
      if (cg_skip(i, gated)) continue;
      R t = fma_(-reg[i], vec[i], accel_divergence(i));
      R v = -(scale * t);
      pair_x[i] = vec[i] * v;
      pair_y[i] = R(0);
      if (bias) v = v - (div ? src[i] : src[i] - R(1));
      if (accumulate) v = v + out[i];
      out[i] = v;
    }
  }

  void cg_sums(bool with_max) {
    world_sum<R>(W, ws.data(), pair_x.data(), sum_x.data(), nullptr);
    world_sum<R>(W, ws.data(), pair_y.data(), sum_y.data(), with_max ? cg_emax.data() : nullptr);
  }

  void cg_solve(bool div, R dt, float tol, float tol_max, int& n_unconv) {
    const R scale = div ? dt : dt * dt;
    const R min_nb = R(P.min_nb);
    auto zr = [&](std::vector<R>& a) { a.assign(n, R(0)); };
    zr(cg_pd); zr(cg_pdr); zr(cg_z); zr(cg_w); zr(cg_ap); zr(cg_corr); zr(cg_corrr); zr(pair_x); zr(pair_y);
    cg_act.assign(n, 0);
    cg_restart.assign(W, 0);
    cg_rz.assign(W, 0.0); cg_step.assign(W, 0.0); sum_x.assign(W, 0.0); sum_y.assign(W, 0.0);
    cg_emax.assign(W, 0.0f);
    // krylov.py:278-285 init: w = A k - b, active set, z = M^-1 r, p = z, r.z
    cg_accel(kappa, kr, false);
    cg_apply(div, dt, kappa, cg_w, false, true, false);
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      const bool a = kappa[i] > lower[i] || cg_w[i] < R(0);
      const R zi = a ? ((-cg_w[i]) * alpha[i]) / scale : R(0);
      cg_act[i] = a ? 1 : 0;
      cg_z[i] = zi;
      cg_pd[i] = zi;
      cg_pdr[i] = zi / R(rho0[i]);
      pair_x[i] = -cg_w[i] * zi;
      pair_y[i] = R(0);
    }
    cg_sums(false);
    for (int w = 0; w < W; ++w) { cg_rz[w] = sum_x[w]; cg_restart[w] = 0; }
    int guard = 0;
    while (n_unconv > 0 && guard++ < 100000) {
      // krylov.py:287-290: Ap and p.Ap
      cg_accel(cg_pd, cg_pdr, false);
      cg_apply(div, dt, cg_pd, cg_ap, false, false, false);
      cg_sums(false);
      // krylov.py:146-170: k += a p on F, projected; w += a Ap
      for (int i = 0; i < n; ++i) {
        if (!is_fluid(i)) { cg_corr[i] = R(0); cg_corrr[i] = R(0); continue; }
        const int w = world[i];
        if (converged[w]) continue;
        double pap = sum_x[w];
        const R a = R(pap > 1.0e-30 ? cg_rz[w] / pap : 0.0);
        R c = R(0);
        if (cg_act[i]) {
          R k = fma_(a, cg_pd[i], kappa[i]);
          if (k < lower[i]) {
            c = lower[i] - k;
            k = lower[i];
            cg_act[i] = 0;
            cg_restart[w] += 1;
          }
          kappa[i] = k;
          kr[i] = k / R(rho0[i]);
        }
        cg_corr[i] = c;
        cg_corrr[i] = c / R(rho0[i]);
        cg_w[i] = fma_(a, cg_ap[i], cg_w[i]);
      }
      // krylov.py:292: w += A c in worlds where something was clamped
      cg_accel(cg_corr, cg_corrr, true);
      cg_apply(div, dt, cg_corr, cg_w, true, false, true);
      // krylov.py:173-204: activation, z, error
      for (int i = 0; i < n; ++i) {
        if (!is_fluid(i)) { pair_x[i] = R(0); pair_y[i] = R(0); err[i] = R(0); continue; }
        const int w = world[i];
        if (converged[w]) continue;
        const R wv = cg_w[i];
        if (!cg_act[i] && wv < R(0)) { cg_act[i] = 1; cg_restart[w] += 1; }
        const R zi = cg_act[i] ? ((-wv) * alpha[i]) / scale : R(0);
        cg_z[i] = zi;
        R e = maxr(-wv, R(0));
        if (kappa[i] > lower[i]) e = std::fabs(wv);
        if (div) {
          if (neff[i] < min_nb) e = R(0);
          e = e * dt;
        }
        err[i] = e;
        pair_x[i] = -wv * zi;
        pair_y[i] = e;
      }
      cg_sums(true);
      // krylov.py:207-233: stop test, beta
      n_unconv = 0;
      for (int w = 0; w < W; ++w) {
        if (converged[w]) continue;
        int it = iters[w] + 1;
        iters[w] = it;
        const double rz_new = sum_x[w];
        float mean = (float)(sum_y[w] / std::max(n_active[w], 1.0));
        err_mean[w] = mean;
        double beta = 0.0;
        if (cg_restart[w] == 0 && cg_rz[w] > 1.0e-30) beta = rz_new / cg_rz[w];
        cg_restart[w] = 0;
        cg_rz[w] = rz_new;
        cg_step[w] = beta;
        const float ts = tol_scale[w];
        if ((it >= P.min_it && mean <= tol * ts && cg_emax[w] <= tol_max * ts) || it >= P.max_it) converged[w] = 1;
        else n_unconv++;
      }
      // krylov.py:236-246: p = z + beta p on F
      for (int i = 0; i < n; ++i) {
        if (!is_fluid(i)) continue;
        const int w = world[i];
        if (converged[w]) continue;
        const R pd = cg_act[i] ? fma_(R(cg_step[w]), cg_pd[i], cg_z[i]) : R(0);
        cg_pd[i] = pd;
        cg_pdr[i] = pd / R(rho0[i]);
      }
    }
  }

  // pressure.py:355-390 + solve_driver.py:121-186 (Jacobi branch)
  void solve(bool div, R dt, double dt_d) {
    const double tol_d = div ? P.tol_div : P.tol_den;
    const float tol = (float)tol_d, tol_max = (float)(tol_d * P.max_error_factor);
    R relief = R(1.0e30);
    if (!div && P.relief_speed > 0.0) relief = R(P.relief_speed * dt_d * P.lattice_grad);
    if (div) tol_scale.assign(W, 1.0f);
    else density_tolerance(dt);
    solve_init(div, dt, relief);
    refresh_kr();
    int n_unconv = 0;
    for (int w = 0; w < W; ++w) {
      iters[w] = 0;
      err_mean[w] = 0.0f;
      if (n_active[w] > 0.0) { converged[w] = 0; n_unconv++; } else converged[w] = 1;
    }
    std::vector<double> esum(W);
    std::vector<float> emax(W);
    int guard = 0;
    if (P.cg) cg_solve(div, dt, tol, tol_max, n_unconv);
    while (!P.cg && n_unconv > 0 && guard++ < 100000) {
      accel_pass();
      jacobi_pass(div, dt);
      world_sum<R>(W, ws.data(), err.data(), esum.data(), emax.data());
      n_unconv = 0;
      for (int w = 0; w < W; ++w) {
        if (converged[w]) continue;
        int it = iters[w] + 1;
        iters[w] = it;
        float mean = (float)(esum[w] / std::max(n_active[w], 1.0));
        err_mean[w] = mean;
        const float ts = tol_scale[w];
        if ((it >= P.min_it && mean <= tol * ts && emax[w] <= tol_max * ts) || it >= P.max_it) converged[w] = 1;
        else n_unconv++;
      }
    }
    contact_limit(dt);
    apply_pressure(div, dt);
    lone_friction(dt);
    for (int w = 0; w < W; ++w) {
      if (div) { iters_div[w] = iters[w]; div_err[w] = err_mean[w]; }
      else { iters_den[w] = iters[w]; den_err[w] = err_mean[w]; }
    }
    if (!div) {
      for (int w = 0; w < W; ++w) { den_err_max[w] = 0.0f; den_tol[w] = tol * tol_scale[w]; }
      for (int i = 0; i < n; ++i)
        if (is_fluid(i)) den_err_max[world[i]] = maxr(den_err_max[world[i]], (float)err[i]);
    }
  }

  // pressure.py:393-414: a lone particle's push may stop its approach and separate it at most v_sep from its walls
  void contact_limit(R dt) {
    const R v_sep = R(P.v_sep);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i) || cnt[i] > 0 || kappa[i] <= R(0)) continue;
      if (s_cnt[i] == 0) continue;
      V3<R> G{R(0), R(0), R(0)}, vb{R(0), R(0), R(0)};
      R ps = R(0);
      for (int b = 0; b < s_cnt[i]; ++b) {
        const size_t o = (size_t)i * NS + b;
        G = {G.x + s_g[o].x, G.y + s_g[o].y, G.z + s_g[o].z};
        vb = {fma_(s_psi[o], s_vb[o].x, vb.x), fma_(s_psi[o], s_vb[o].y, vb.y), fma_(s_psi[o], s_vb[o].z, vb.z)};
        ps = ps + s_psi[o];
      }
      R g = std::sqrt(dot_plain(G, G));
      if (g <= R(0)) continue;
      if (ps > R(0)) vb = {vb.x / ps, vb.y / ps, vb.z / ps};
      V3<R> nn{-G.x / g, -G.y / g, -G.z / g};
      R u = dotf(sub(v[i], vb), nn);
      kappa[i] = minr(kappa[i], maxr(v_sep - u, R(0)) / (dt * g));
    }
  }

  // pressure.py:417-458: Coulomb friction of a lone particle on its walls, after the solve's velocity update: the
  // wall's push dv_n = dt k |G| takes up to mu dv_n of its tangential speed relative to the walls, never reversing
  // it; mu is that of the wall in its largest-Psi slot (a particle wall has none)
  void lone_friction(R dt) {
    if (!P.wall_friction || S == 0) return;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i) || cnt[i] > 0 || kappa[i] <= R(0) || s_cnt[i] == 0) continue;
      V3<R> G{R(0), R(0), R(0)}, vb{R(0), R(0), R(0)};
      R ws = R(0), pbest = R(0);
      int best = -1;
      for (int b = 0; b < s_cnt[i]; ++b) {
        const size_t o = (size_t)i * NS + b;
        G = {G.x + s_g[o].x, G.y + s_g[o].y, G.z + s_g[o].z};
        vb = {fma_(s_psi[o], s_vb[o].x, vb.x), fma_(s_psi[o], s_vb[o].y, vb.y), fma_(s_psi[o], s_vb[o].z, vb.z)};
        ws = ws + s_psi[o];
        if (s_psi[o] > pbest) { pbest = s_psi[o]; best = b; }
      }
      R g = std::sqrt(dot_plain(G, G));
      if (g <= R(0) || ws <= R(0) || best < 0) continue;
      const int sh = s_shape[(size_t)i * NS + best];
      if (sh >= S) continue;
      const R mu = R(sh_mu[sh]);
      if (mu <= R(0)) continue;
      const V3<R> nn{-G.x / g, -G.y / g, -G.z / g};
      const V3<R> u = sub(v[i], V3<R>{vb.x / ws, vb.y / ws, vb.z / ws});
      const R un = dotf(u, nn);
      const V3<R> vt{fma_(-un, nn.x, u.x), fma_(-un, nn.y, u.y), fma_(-un, nn.z, u.z)};
      const R lt = std::sqrt(dot_plain(vt, vt));
      if (lt <= R(0)) continue;
      const R f = minr(R(1), (((mu * dt) * kappa[i]) * g) / lt);
      v[i] = {fma_(-f, vt.x, v[i].x), fma_(-f, vt.y, v[i].y), fma_(-f, vt.z, v[i].z)};
    }
  }

  // pressure.py:461-480 (slot impulses are coupling output and not tracked here)
  void apply_pressure(bool div, R dt) {
    refresh_kr();
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      V3<R> a = pressure_accel(i, kr);
      acc[i] = a;
    }
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      v[i] = {fma_(dt, acc[i].x, v[i].x), fma_(dt, acc[i].y, v[i].y), fma_(dt, acc[i].z, v[i].z)};
      if (div) kv[i] = kappa[i] * dt;
      else kd[i] = (kappa[i] * dt) * dt;
    }
  }

  // integrate.py:150-178
  void nonpressure(R dt) {
    const R c = R(P.xsph_c);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < n; ++i) {
      V3<R> vi = v[i];
      if (!is_fluid(i)) { vtmp[i] = vi; continue; }
      int w = world[i];
      V3<R> g{R(gravity[3 * w]), R(gravity[3 * w + 1]), R(gravity[3 * w + 2])};
      V3<R> vn{fma_(dt, g.x, vi.x), fma_(dt, g.y, vi.y), fma_(dt, g.z, vi.z)};
      if (c > R(0)) {
        const V3<R> xi = q[i];
        V3<R> corr{R(0), R(0), R(0)};
        R rho_i = ratio[i] * R(rho0[i]);
        const int* row = &nbr[(size_t)i * K];
        for (int k = 0; k < cnt[i]; ++k) {
          int j = row[k];
          R rho_bar = R(0.5) * (rho_i + ratio[j] * R(rho0[j]));
          if (rho_bar > R(0)) {
            V3<R> rv = sub(xi, q[j]);
            R Wv, F;
            wf(kc, dot_plain(rv, rv), Wv, F);
            R cw = (R(mass[j]) / rho_bar) * Wv;
            corr.x = fma_(cw, v[j].x - vi.x, corr.x);
            corr.y = fma_(cw, v[j].y - vi.y, corr.y);
            corr.z = fma_(cw, v[j].z - vi.z, corr.z);
          }
        }
        vn = {fma_(c, corr.x, vn.x), fma_(c, corr.y, vn.y), fma_(c, corr.z, vn.z)};
      }
      vtmp[i] = vn;
    }
    v.swap(vtmp);
  }

  // integrate.py:75-95 (box_span) and 98-126 (path_entry) for a static box: the last outside parameter of the path
  // l0 -> l1 (its frame) before it first enters box sh, by the exact slab test; 2 when it stays outside or starts
  // inside
  R box_entry(int sh, const V3<R>& l0, const V3<R>& l1) const {
    const float* hx = &sh_half[3 * sh];
    if (box_sdf(l0, hx) < R(0)) return R(2);
    R lo = R(-1.0e30), hi = R(1.0e30);
    const R d[3] = {l1.x - l0.x, l1.y - l0.y, l1.z - l0.z}, o[3] = {l0.x, l0.y, l0.z};
    for (int a = 0; a < 3; ++a) {
      const R h = R(hx[a]);
      if (std::fabs(d[a]) > R(0)) {
        const R ta = (-h - o[a]) / d[a], tb = (h - o[a]) / d[a];
        lo = maxr(lo, minr(ta, tb));
        hi = minr(hi, maxr(ta, tb));
      } else if (std::fabs(o[a]) > h) {
        lo = R(2.0e30);
      }
    }
    if (lo <= hi && lo <= R(1) && hi >= R(0)) return maxr(lo, R(0));
    return R(2);
  }

  // integrate.py:48-58 and 98-115 (path_entry) for a shape other than a box: the path l0 -> l1 sampled at `samples`
  // evenly spaced parameters, the first sample inside and the last before it bisected 8 times; the last outside
  // parameter, or 2 when the path stays outside or starts inside
  R shape_entry(int sh, const V3<R>& l0, const V3<R>& l1, int samples) const {
    if (sh_geo[sh] == GEO_BOX) return box_entry(sh, l0, l1);
    if (shape_phi(sh, l0) < R(0)) return R(2);
    const V3<R> d{l1.x - l0.x, l1.y - l0.y, l1.z - l0.z};
    auto inside = [&](R t) { return shape_phi(sh, V3<R>{fma_(t, d.x, l0.x), fma_(t, d.y, l0.y), fma_(t, d.z, l0.z)}) < R(0); };
    R t_lo = R(0), t_hi = R(2);
    for (int k = 1; k <= samples && t_hi > R(1); ++k) {
      const R t = R(k) / R(samples);
      if (inside(t)) t_hi = t;
      else t_lo = t;
    }
    if (t_hi > R(1)) return R(2);
    for (int b = 0; b < 8; ++b) {
      const R tm = R(0.5) * (t_lo + t_hi);
      if (inside(tm)) t_hi = tm;
      else t_lo = tm;
    }
    return t_lo;
  }

  // integrate.py:192-205: Coulomb friction of a projection (Config.wall_friction) after the inward speed -vn went
  V3<R> wall_friction_v(V3<R> vv, const V3<R>& vb, const V3<R>& nn, R vn, int sh) const {
    if (!P.wall_friction) return vv;
    const R mu = R(sh_mu[sh]);
    if (mu <= R(0)) return vv;
    const V3<R> u = sub(vv, vb);
    const R un = dotf(u, nn);
    const V3<R> vt{fma_(-un, nn.x, u.x), fma_(-un, nn.y, u.y), fma_(-un, nn.z, u.z)};
    const R lt = std::sqrt(dot_plain(vt, vt));
    if (lt <= R(0)) return vv;
    const R f = minr(R(1), (mu * (-vn)) / lt);
    return {fma_(-f, vt.x, vv.x), fma_(-f, vt.y, vv.y), fma_(-f, vt.z, vv.z)};
  }

  // integrate.py:181-185 + particle_walls.py:131-135 + integrate.py:212-309: advection, then each liquid particle
  // that moved further than the sweep length is swept along its path against its world's walls, and its slots'
  // walls push it out in up to PROJECT_PASSES passes (the particle wall onto its start plane advanced with the wall;
  // a box through its SDF at the new place, onto its start-of-step tangent plane when that holds it)
  void advect_project(R dt) {
    const R eps = R(P.project_eps), r = R(P.particle_radius), sweep = R(sweep_len);
    std::vector<int> moved_w(W, 0), swept_w(W, 0);
    for (int i = 0; i < n; ++i) {
      if (is_fluid(i)) {
        q[i] = {fma_(dt, v[i].x, q[i].x), fma_(dt, v[i].y, q[i].y), fma_(dt, v[i].z, q[i].z)};
      } else if (wall_vol[i] > 0.0f) {
        q[i] = {fma_(dt, v[i].x, q[i].x), fma_(dt, v[i].y, q[i].y), fma_(dt, v[i].z, q[i].z)};
      }
    }
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      const int w = world[i];
      V3<R> x = q[i], vv = v[i];
      int moved = 0;
      const V3<R> step{dt * vv.x, dt * vv.y, dt * vv.z};
      if (sh_start[w + 1] > sh_start[w] && std::sqrt(dot_plain(step, step)) > sweep) {
        const V3<R> x0{x.x - step.x, x.y - step.y, x.z - step.z};
        const V3<R> span = sub(x, x0);
        const R len = std::sqrt(dot_plain(span, span));
        const R reach = len + r;
        const int samples = std::min(std::max((int)std::ceil(len / r) + 1, 8), 64);  // integrate.py:48, 56-58
        R best = R(2);
        int hit = -1;
        V3<R> lh{R(0), R(0), R(0)};
        for (int c = sh_start[w]; c < sh_start[w + 1]; ++c) {
          const int sh = sh_ids[c];
          const V3<R> d0{x0.x - R(sh_pos[3 * sh]), x0.y - R(sh_pos[3 * sh + 1]), x0.z - R(sh_pos[3 * sh + 2])};
          if (sh_geo[sh] != GEO_PLANE && !(std::sqrt(dot_plain(d0, d0)) <= R(sh_radius[sh]) + reach)) continue;
          const V3<R> l0 = shape_local(sh, x0), l1 = shape_local(sh, x);
          const R t = shape_entry(sh, l0, l1, samples);
          if (t < best) {
            best = t;
            hit = sh;
            lh = {fma_(t, l1.x - l0.x, l0.x), fma_(t, l1.y - l0.y, l0.y), fma_(t, l1.z - l0.z, l0.z)};
          }
        }
        if (hit >= 0) {
          const R phi = shape_phi(hit, lh);
          const V3<R> nn = from_frame(hit, normalized(shape_grad(hit, lh)));
          const V3<R> xw = shape_world(hit, from_frame(hit, lh));
          const R push = maxr(eps - phi, R(0));
          x = {fma_(push, nn.x, xw.x), fma_(push, nn.y, xw.y), fma_(push, nn.z, xw.z)};
          const R vn = dotf(vv, nn);
          if (vn < R(0)) {
            vv = {fma_(-vn, nn.x, vv.x), fma_(-vn, nn.y, vv.y), fma_(-vn, nn.z, vv.z)};
            vv = wall_friction_v(vv, V3<R>{R(0), R(0), R(0)}, nn, vn, hit);
          }
          moved = 1;
          swept_w[w]++;
        }
      }
      int busy = 1;
      for (int pass = 0; pass < PROJECT_PASSES && busy; ++pass) {
        busy = 0;
        for (int b = 0; b < s_cnt[i]; ++b) {
          const size_t o = (size_t)i * NS + b;
          const int sh = s_shape[o];
          if (sh == S) {  // the particle wall's plane at its end-of-step place
            const V3<R> nn = s_nbl[o], vb = s_vb[o], xb = s_xbl[o];
            const V3<R> pp{fma_(dt, vb.x, xb.x), fma_(dt, vb.y, xb.y), fma_(dt, vb.z, xb.z)};
            const R d = dotf(sub(x, pp), nn);
            if (d < eps) {
              const R push = eps - d;
              x = {fma_(push, nn.x, x.x), fma_(push, nn.y, x.y), fma_(push, nn.z, x.z)};
              const R vn = dotf(sub(vv, vb), nn);
              if (vn < R(0)) vv = {fma_(-vn, nn.x, vv.x), fma_(-vn, nn.y, vv.y), fma_(-vn, nn.z, vv.z)};
              moved = busy = 1;
            }
          } else if (sh >= 0) {  // a static shape: its SDF at the new place, its start plane when that holds it
            const V3<R> xl = shape_local(sh, x);
            const R phi = shape_phi(sh, xl);
            if (phi < eps) {
              V3<R> nn = from_frame(sh, normalized(shape_grad(sh, xl)));
              R push = eps - phi;
              if (s_phi[o] >= R(0)) {
                const V3<R> ns = s_nbl[o];
                const R push_s = eps - dotf(ns, sub(x, shape_world(sh, s_xbl[o])));
                if (push_s > R(0)) { nn = ns; push = push_s; }
              }
              if (push > R(0)) {
                x = {fma_(push, nn.x, x.x), fma_(push, nn.y, x.y), fma_(push, nn.z, x.z)};
                const R vn = dotf(vv, nn);
                if (vn < R(0)) {
                  vv = {fma_(-vn, nn.x, vv.x), fma_(-vn, nn.y, vv.y), fma_(-vn, nn.z, vv.z)};
                  vv = wall_friction_v(vv, V3<R>{R(0), R(0), R(0)}, nn, vn, sh);
                }
                moved = busy = 1;
              }
            }
          }
        }
      }
      if (moved) { q[i] = x; v[i] = vv; moved_w[w]++; }
    }
    for (int w = 0; w < W; ++w) { projected[w] += moved_w[w]; swept[w] += swept_w[w]; }
  }

  // emitters.py:134-164
  void retire() {
    bool any = P.has_bounds || !sinks.empty();
    if (!any) return;
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      int w = world[i];
      V3<R> x = q[i];
      int gone = 0;
      for (const Sink& s : sinks) {
        if (s.world != w) continue;
        V3<R> d{x.x - R(s.xform[0]), x.y - R(s.xform[1]), x.z - R(s.xform[2])};
        float inv[4] = {-s.xform[3], -s.xform[4], -s.xform[5], s.xform[6]};
        V3<R> xl = quat_rotate(inv, d);
        if (std::fabs(xl.x) <= R(s.half[0]) && std::fabs(xl.y) <= R(s.half[1]) && std::fabs(xl.z) <= R(s.half[2])) gone = 1;
      }
      if (P.has_bounds && gone == 0) {
        bool out = x.x < R(P.bounds_lo[0]) || x.y < R(P.bounds_lo[1]) || x.z < R(P.bounds_lo[2]) ||
                   x.x > R(P.bounds_hi[0]) || x.y > R(P.bounds_hi[1]) || x.z > R(P.bounds_hi[2]);
        if (out || !std::isfinite((x.x + x.y) + x.z)) { gone = 2; escaped[w]++; }
      }
      if (gone) {
        flags[i] &= ~FLAG_ACTIVE;
        phase[i] = -2;
        v[i] = {R(0), R(0), R(0)};
        mass_out[w] += to_fixed(mass[i]);
      }
    }
  }

  // emitters.py:67-126
  void emit(R dt) {
    for (Emitter& e : emitters) {
      int now = 0;
      if (e.enabled) {
        float t = e.t_acc + (float)dt;
        if (t >= e.interval) { t -= e.interval; now = 1; }
        e.t_acc = t;
      }
      if (!now) continue;
      int nl = (int)(e.offsets.size() / 3);
      for (int c = 0; c < nl; ++c) {
        int slot = e.cursor + c;
        if (slot >= (int)e.pool.size()) { emit_overflow[e.world]++; continue; }
        int i = e.pool[slot];
        V3<R> p{R(e.offsets[3 * c]), R(e.offsets[3 * c + 1]), R(e.offsets[3 * c + 2])};
        V3<R> r = quat_rotate(e.xform + 3, p);
        q[i] = {r.x + R(e.xform[0]), r.y + R(e.xform[1]), r.z + R(e.xform[2])};
        v[i] = {R(e.vel[0]), R(e.vel[1]), R(e.vel[2])};
        flags[i] |= FLAG_ACTIVE;
        phase[i] = 1;
        mass_in[e.world] += to_fixed(mass[i]);
      }
      e.cursor = std::min(e.cursor + nl, (int)e.pool.size());
    }
  }

  // integrate.py:312-326
  void speed() {
    for (int w = 0; w < W; ++w) max_speed[w] = 0.0f;
    for (int i = 0; i < n; ++i) {
      if (!is_fluid(i)) continue;
      int w = world[i];
      R s = std::sqrt(dotf(v[i], v[i]));
      V3<R> x = q[i];
      if (std::isfinite(s) && std::isfinite((x.x + x.y) + x.z)) max_speed[w] = maxr(max_speed[w], (float)s);
      else { nonfinite[w]++; max_speed[w] = maxr(max_speed[w], 1.0e30f); }
    }
  }

  void prepare_density() {
    build_groups_and_grids();
    build_lists();
    wall_slots();
    density_alpha();
    for (int w = 0; w < W; ++w) {
      double a = 0.0;
      for (int i = ws[w]; i < ws[w + 1]; ++i) a += (double)active[i];
      n_active[w] = a;
    }
  }

  // prime.py:52-87: the hydrostatic pressure of a fluid at rest. The caller stores the hydrostatic guess as the
  // divergence warm start (kv = guess dt); one divergence solve (tolerance tol, up to max_it iterations, plain
  // start 1 x kv, no neighbour floor, no max-error test) of the velocity one gravity step adds; velocities are left
  // unchanged; the density warm start becomes kd = kv dt and kv is cleared. Returns the iterations used.
  int prime(double dt_d, double tol, int max_it) {
    R dt = R(dt_d);
    const std::vector<V3<R>> v_saved = v;
    const OrcParams saved = P;
    prepare_density();
    nonpressure(dt);
    P.tol_div = tol;
    P.max_it = max_it;
    P.warm_div = 1.0;
    P.min_nb = 0.0;
    P.max_error_factor = 1.0e9;
    solve(true, dt, dt_d);
    P = saved;
    v = v_saved;
    for (int i = 0; i < n; ++i) {
      kd[i] = kv[i] * dt;
      kv[i] = R(0);
    }
    int it = 0;
    for (int w = 0; w < W; ++w) it = std::max(it, iters_div[w]);
    return it;
  }

  // solve_driver.py:38-51 (_flow_speed): the per-world float64 sums of the liquid's start velocity (v_z, 1, v_x, v_y)
  // in world_sum's tree order, when the rule and its flow ratio are on
  void flow_sums() {
    if (!(P.jitter_speed > 0.0) || !(P.jitter_ratio > 0.0)) return;
    std::vector<R> t(n);
    for (int k = 0; k < 4; ++k) {
      for (int i = 0; i < n; ++i)
        t[i] = !is_fluid(i) ? R(0) : k == 0 ? v[i].z : k == 1 ? R(1) : k == 2 ? v[i].x : v[i].y;
      flow_sum[k].assign(W, 0.0);
      world_sum<R>(W, ws.data(), t.data(), flow_sum[k].data(), nullptr);
    }
  }

  // solve_driver.py:54-110 (_density_tolerance, tol_scale_kernel): per world the factor of the density solve's
  // tolerance, clamp(v dt / (H tol), tol_min / tol, 1), H = 1.5 S2 / (S1 dt^2 |g|) from the density warm starts
  // (S1 = sum kd+, S2 = sum kd+^2 over the liquid, kd+ = max(kd, 0)), v = max(speed, ratio |mean velocity|); float32
  // arithmetic as the kernel's
  void density_tolerance(R dt) {
    tol_scale.assign(W, 1.0f);
    if (!(P.jitter_speed > 0.0)) return;
    std::vector<R> t1(n), t2(n);
    for (int i = 0; i < n; ++i) {
      const R k = is_fluid(i) ? maxr(kd[i], R(0)) : R(0);
      t1[i] = k;
      t2[i] = k * k;
    }
    std::vector<double> s1(W), s2(W);
    world_sum<R>(W, ws.data(), t1.data(), s1.data(), nullptr);
    world_sum<R>(W, ws.data(), t2.data(), s2.data(), nullptr);
    const float fdt = (float)dt, speed = (float)P.jitter_speed, ratio = (float)P.jitter_ratio;
    const float tol = (float)P.tol_den, tol_min = (float)P.tol_den_min;
    for (int w = 0; w < W; ++w) {
      float sc = 1.0f;
      const float gx = gravity[3 * w], gy = gravity[3 * w + 1], gz = gravity[3 * w + 2];
      const float g = std::sqrt((gx * gx + gy * gy) + gz * gz);
      const float a = (float)s1[w], b = (float)s2[w];
      float vs = speed;
      if (ratio > 0.0f && !flow_sum[1].empty() && flow_sum[1][w] > 0.0) {
        const double cnt = flow_sum[1][w];
        const float ux = (float)(flow_sum[2][w] / cnt), uy = (float)(flow_sum[3][w] / cnt);
        const float uz = (float)(flow_sum[0][w] / cnt);
        vs = maxr(vs, ratio * std::sqrt((ux * ux + uy * uy) + uz * uz));
      }
      if (g > 0.0f && a > 0.0f && b > 0.0f) {
        const float depth = (1.5f * b) / (((a * fdt) * fdt) * g);
        sc = minr(maxr((vs * fdt) / (depth * tol), tol_min / tol), 1.0f);
      }
      tol_scale[w] = sc;
    }
  }

  // solver.py:218-268
  void step(double dt_d) {
    R dt = R(dt_d);
    prepare_density();
    flow_sums();
    if (P.divergence_solve) solve(true, dt, dt_d);
    nonpressure(dt);
    solve(false, dt, dt_d);
    advect_project(dt);
    retire();
    emit(dt);
    speed();
  }
};

struct Handle {
  int f64;
  std::unique_ptr<Solver<float>> s32;
  std::unique_ptr<Solver<double>> s64;
};

template <class R> void setup(Solver<R>& s, const OrcParams* p, int n, int W, const int* ws, const float* mass,
                               const float* rho0, const int* flags, const int8_t* phase, const int* world,
                               const float* wall_vol, const float* gravity) {
  s.P = *p;
  s.n = n;
  s.W = W;
  s.ws.assign(ws, ws + W + 1);
  s.mass.assign(mass, mass + n);
  s.rho0.assign(rho0, rho0 + n);
  s.flags.assign(flags, flags + n);
  s.phase.assign(phase, phase + n);
  s.world.assign(world, world + n);
  s.wall_vol.assign(wall_vol, wall_vol + n);
  s.gravity.assign(gravity, gravity + 3 * W);
  s.init();
  s.init_mass();
#ifdef _OPENMP
  s.nthreads = omp_get_max_threads();
#endif
}

template <class R, class T> void copy_out(const std::vector<R>& a, T* out) {
  for (size_t i = 0; i < a.size(); ++i) out[i] = (T)a[i];
}
template <class R, class T> void copy_out3(const std::vector<V3<R>>& a, T* out) {
  for (size_t i = 0; i < a.size(); ++i) { out[3 * i] = (T)a[i].x; out[3 * i + 1] = (T)a[i].y; out[3 * i + 2] = (T)a[i].z; }
}

}  // namespace

extern "C" {

typedef OrcParams orc_params;

void* orc_create(const orc_params* p, int n, int W, const int* ws, const float* mass, const float* rho0,
                 const int* flags, const int8_t* phase, const int* world, const float* wall_vol, const float* gravity,
                 int f64) {
  Handle* h = new Handle();
  h->f64 = f64;
  if (f64) { h->s64.reset(new Solver<double>()); setup(*h->s64, p, n, W, ws, mass, rho0, flags, phase, world, wall_vol, gravity); }
  else { h->s32.reset(new Solver<float>()); setup(*h->s32, p, n, W, ws, mass, rho0, flags, phase, world, wall_vol, gravity); }
  return h;
}

void orc_destroy(void* hp) { delete (Handle*)hp; }

void orc_set_threads(void* hp, int t) {
  Handle* h = (Handle*)hp;
  if (h->f64) h->s64->nthreads = t; else h->s32->nthreads = t;
}

#define DISPATCH(...) do { Handle* h = (Handle*)hp; if (h->f64) { auto& s = *h->s64; __VA_ARGS__; } else { auto& s = *h->s32; __VA_ARGS__; } } while (0)

void orc_set_state(void* hp, const float* q, const float* qd) {
  DISPATCH({
    using R = typename std::remove_reference<decltype(s.kv)>::type::value_type;
    for (int i = 0; i < s.n; ++i) {
      s.q[i] = {R(q[3 * i]), R(q[3 * i + 1]), R(q[3 * i + 2])};
      s.v[i] = {R(qd[3 * i]), R(qd[3 * i + 1]), R(qd[3 * i + 2])};
    }
  });
}
// Velocities of m particles (kinematic walls driven by the caller between steps), in the working precision.
void orc_set_velocity(void* hp, int m, const int* idx, const float* v) {
  DISPATCH({
    using R = typename std::remove_reference<decltype(s.kv)>::type::value_type;
    for (int k = 0; k < m; ++k) s.v[idx[k]] = {R(v[3 * k]), R(v[3 * k + 1]), R(v[3 * k + 2])};
  });
}
void orc_get_state(void* hp, float* q, float* qd) { DISPATCH({ copy_out3(s.q, q); copy_out3(s.v, qd); }); }
void orc_get_state_f64(void* hp, double* q, double* qd) { DISPATCH({ copy_out3(s.q, q); copy_out3(s.v, qd); }); }
void orc_set_warm(void* hp, const float* kv, const float* kd) {
  DISPATCH({
    for (int i = 0; i < s.n; ++i) { s.kv[i] = kv[i]; s.kd[i] = kd[i]; }
  });
}
void orc_get_warm(void* hp, float* kv, float* kd) { DISPATCH({ copy_out(s.kv, kv); copy_out(s.kd, kd); }); }
void orc_get_flags_phase(void* hp, int* flags, int8_t* phase) {
  DISPATCH({
    std::memcpy(flags, s.flags.data(), sizeof(int) * s.n);
    std::memcpy(phase, s.phase.data(), s.n);
  });
}
int orc_step(void* hp, double dt) { DISPATCH(s.step(dt)); return 0; }
int orc_prime(void* hp, double dt, double tol, int max_it) {
  int it = 0;
  DISPATCH(it = s.prime(dt, tol, max_it));
  return it;
}
void orc_prepare_density(void* hp) { DISPATCH(s.prepare_density()); }

// name: ratio alpha neff active reg src kappa err, and slot k's (k = 0 when the name has no suffix, else the digit
// after a colon, e.g. "slot_psi:1") slot_psi slot_phi slot_g slot_vb slot_n
int orc_get_field(void* hp, const char* name, float* out) {
  int ok = 1;
  DISPATCH({
    auto pick = [&](const char* nm, const auto& a) { if (std::strcmp(name, nm) == 0) { copy_out(a, out); ok = 0; } };
    pick("ratio", s.ratio); pick("alpha", s.alpha); pick("neff", s.neff); pick("active", s.active);
    pick("reg", s.reg); pick("src", s.src); pick("kappa", s.kappa); pick("err", s.err);
    if (std::strcmp(name, "acc") == 0) { copy_out3(s.acc, out); ok = 0; }
    const char* colon = std::strchr(name, ':');
    const size_t base = colon ? (size_t)(colon - name) : std::strlen(name);
    const int k = colon ? std::atoi(colon + 1) : 0;
    auto is = [&](const char* nm) { return std::strlen(nm) == base && std::strncmp(name, nm, base) == 0; };
    if (k >= 0 && k < NS) {
      for (int i = 0; i < s.n; ++i) {
        const size_t o = (size_t)i * NS + k;
        if (is("slot_psi")) out[i] = (float)s.s_psi[o];
        if (is("slot_phi")) out[i] = (float)s.s_phi[o];
        const auto* v3 = is("slot_g") ? &s.s_g : is("slot_vb") ? &s.s_vb : is("slot_n") ? &s.s_nbl : nullptr;
        if (v3) {
          out[3 * i] = (float)(*v3)[o].x;
          out[3 * i + 1] = (float)(*v3)[o].y;
          out[3 * i + 2] = (float)(*v3)[o].z;
        }
      }
      if (is("slot_psi") || is("slot_phi") || is("slot_g") || is("slot_vb") || is("slot_n")) ok = 0;
    }
  });
  return ok;
}

// per particle: its slot count (0: none), and with shapes != NULL its slots' wall ids [n][4] (-1 empty; the
// particle wall is the shape count)
void orc_get_slot_on(void* hp, int* out) { DISPATCH(std::memcpy(out, s.s_cnt.data(), sizeof(int) * s.n)); }
void orc_get_slot_shapes(void* hp, int* out) {
  DISPATCH(std::memcpy(out, s.s_shape.data(), sizeof(int) * (size_t)s.n * NS));
}

// The liquid's static axis-aligned box walls (layout.py:207-246): S shapes, per-world CSR start[W + 1] / ids, each
// box's centre pos[S][3], half extents half[S][3], bounding radius[S] and friction mu[S]; sweep length
// min(h / 2, thinnest / 2) (integrate.py:42-49).
void orc_set_shapes(void* hp, int S, const int* start, const int* ids, const float* pos, const float* half,
                    const float* radius, const float* mu, double thinnest, const int* geo, const float* quat) {
  DISPATCH({
    s.S = S;
    s.sh_geo.assign(S, 7);
    if (geo) s.sh_geo.assign(geo, geo + S);
    s.sh_quat.assign(4 * (size_t)S, 0.0f);
    for (int k = 0; k < S; ++k) s.sh_quat[4 * (size_t)k + 3] = 1.0f;
    if (quat) s.sh_quat.assign(quat, quat + 4 * (size_t)S);
    s.sh_start.assign(start, start + s.W + 1);
    s.sh_ids.assign(ids, ids + start[s.W]);
    s.sh_pos.assign(pos, pos + 3 * S);
    s.sh_half.assign(half, half + 3 * S);
    s.sh_radius.assign(radius, radius + S);
    s.sh_mu.assign(mu, mu + S);
    s.sweep_len = std::min(0.5 * s.P.h, 0.5 * thinnest);
  });
}

// The signed distance and outward unit gradient of shape sh at shape-local point p (out: phi, gx, gy, gz), as the
// slots, the sweep and the projection evaluate it.
void orc_shape_sdf(void* hp, int sh, const double* p, double* out) {
  DISPATCH({
    using RT = typename std::remove_reference<decltype(s.kv)>::type::value_type;
    const V3<RT> x{RT(p[0]), RT(p[1]), RT(p[2])};
    const V3<RT> g = s.shape_grad(sh, x);
    out[0] = (double)s.shape_phi(sh, x);
    out[1] = (double)g.x;
    out[2] = (double)g.y;
    out[3] = (double)g.z;
  });
}

void orc_get_lists(void* hp, int* rows, int* count) {
  DISPATCH({
    std::memcpy(count, s.cnt.data(), sizeof(int) * s.n);
    for (int i = 0; i < s.n; ++i)
      for (int k = 0; k < s.K; ++k) rows[(size_t)i * s.K + k] = (k < s.cnt[i]) ? s.nbr[(size_t)i * s.K + k] : -1;
  });
}

// int arrays: iters_den iters_div overflow escaped projected nonfinite emit_overflow swept
// float arrays: den_err div_err den_err_max max_speed den_tol ; int64: mass_in mass_out mass0
void orc_get_report(void* hp, int* ints /*8*W*/, float* floats /*5*W*/, int64_t* ledger /*3*W*/) {
  DISPATCH({
    int W = s.W;
    const std::vector<int>* ia[8] = {&s.iters_den, &s.iters_div, &s.overflow, &s.escaped, &s.projected, &s.nonfinite,
                                     &s.emit_overflow, &s.swept};
    for (int k = 0; k < 8; ++k) std::memcpy(ints + k * W, ia[k]->data(), sizeof(int) * W);
    const std::vector<float>* fa[5] = {&s.den_err, &s.div_err, &s.den_err_max, &s.max_speed, &s.den_tol};
    for (int k = 0; k < 5; ++k) std::memcpy(floats + k * W, fa[k]->data(), sizeof(float) * W);
    std::memcpy(ledger, s.mass_in.data(), 8 * W);
    std::memcpy(ledger + W, s.mass_out.data(), 8 * W);
    std::memcpy(ledger + 2 * W, s.mass0.data(), 8 * W);
  });
}

void orc_active_mass(void* hp, int64_t* out) {
  DISPATCH({
    for (int w = 0; w < s.W; ++w) out[w] = 0;
    for (int i = 0; i < s.n; ++i) if (s.is_fluid(i)) out[s.world[i]] += to_fixed(s.mass[i]);
  });
}

void orc_add_emitter(void* hp, int world, const float* xform, const float* offsets, int n_off, const float* vel,
                     float interval, const int* pool, int pool_size) {
  Emitter e;
  e.world = world;
  std::memcpy(e.xform, xform, sizeof(float) * 7);
  std::memcpy(e.vel, vel, sizeof(float) * 3);
  e.interval = interval;
  e.offsets.assign(offsets, offsets + 3 * n_off);
  e.pool.assign(pool, pool + pool_size);
  DISPATCH(s.emitters.push_back(e));
}

void orc_add_sink(void* hp, int world, const float* xform, const float* half) {
  Sink k;
  k.world = world;
  std::memcpy(k.xform, xform, sizeof(float) * 7);
  std::memcpy(k.half, half, sizeof(float) * 3);
  DISPATCH(s.sinks.push_back(k));
}

// ---- scalar primitives and the reducer, for known-answer tests
void orc_kernel_wf(int kind, double h, double sigma, int m, const float* r2, float* Wout, float* Fout) {
  KC<float> k;
  k.init(kind, h, sigma);
  for (int i = 0; i < m; ++i) wf(k, r2[i], Wout[i], Fout[i]);
}
void orc_kernel_wf64(int kind, double h, double sigma, int m, const double* r2, double* Wout, double* Fout) {
  KC<double> k;
  k.init(kind, h, sigma);
  for (int i = 0; i < m; ++i) wf(k, r2[i], Wout[i], Fout[i]);
}
void orc_halfspace(int kind, double h, int m, const float* d, float* psi, float* dpsi) {
  KC<float> k;
  k.init(kind, h, 1.0);
  for (int i = 0; i < m; ++i) halfspace(k, d[i], psi[i], dpsi[i]);
}
void orc_halfspace64(int kind, double h, int m, const double* d, double* psi, double* dpsi) {
  KC<double> k;
  k.init(kind, h, 1.0);
  for (int i = 0; i < m; ++i) halfspace(k, d[i], psi[i], dpsi[i]);
}
void orc_colour_distance(int kind, double h, int m, const float* c, float* out) {
  KC<float> k;
  k.init(kind, h, 1.0);
  for (int i = 0; i < m; ++i) out[i] = colour_distance(k, c[i]);
}
void orc_world_sum(int W, const int* ws, const float* v, double* out, float* out_max) {
  world_sum<float>(W, ws, v, out, out_max);
}

}  // extern "C"
