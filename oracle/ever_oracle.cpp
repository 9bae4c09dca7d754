// EVER exact ellipsoid tracer: CPU oracle.
//
// TEST INFRASTRUCTURE ONLY. This file is a CPU restatement of the reference's
// trace path, used by tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline as the checker. Nothing in the product library links or calls it.
//
// What it restates (paths inside the N-Demir/ever tree):
//   ray setup                 splinetracers/fast_ellipsoid_splinetracer/slang/shaders.slang:178-182
//   ray/ellipsoid roots       slang/tri-intersect.slang:115-131, :164-175; safe-math.slang:238-244
//   entry/exit reporting      slang/shaders.slang:84-107 (intersection) and :117-164 (any-hit k-buffer)
//   round loop / termination  slang/shaders.slang:171-235 (BUFFER_SIZE 16, LOG_CUTOFF 5.54, 1e9 sentinel)
//   event -> control point    slang/shaders.slang:65-82 (+-density, colour from SH)
//   state update              slang/spline-machine.slang:103-138, extract_color :146-154
//   safe math                 splinetracers/slang/safe-math.slang:68-144, tukey_power_ladder :246-253
//   SH basis                  splinetracers/slang/sh.slang:17-103
//   initial density           initialize_density.cu:107-150 (rays that start inside ellipsoids)
//   backward semantics        slang/backwards_kernel.slang:259-367 (zero gradient when iters >= max_iters-1)
//
// The float32 path ("f32") fixes one exact operation order (explicit fma where the
// CUDA kernels use fma, nothing contracted otherwise; build with -ffp-contract=off).
// Event times, event order, iteration counts and the density sums that drive
// termination are therefore bit-identical to the CUDA kernels; colours differ only by
// the last-bit differences of expf/powf between libm and CUDA.
// The float64 path ("f64") runs the same algorithm in double for the FP64 error
// figures, the analytic backward and central finite differences.
//
// Ties between different ellipsoids at exactly equal t are ordered by ellipsoid index
// here; the reference orders them by OptiX traversal order (unpinned).

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

template <class T> struct K;
template <> struct K<float> {
  static constexpr float tiny = 1.0754944e-20f;  // safe-math.slang:16
  static constexpr float maxv = 1e20f;           // safe-math.slang:18
  static constexpr float minv = -1e20f;          // safe-math.slang:17
  static constexpr float logmax = 46.05170185988091f;
  static constexpr float c0 = 0.28209479177387814f;
  static constexpr float c1 = 0.4886025119029199f;
  static constexpr float c2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                                   -1.0925484305920792f, 0.5462742152960396f};
  static constexpr float c3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                                  0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                                  -0.5900435899266435f};
};
template <> struct K<double> {
  static constexpr double tiny = 1.0754944e-20;
  static constexpr double maxv = 1e20;
  static constexpr double minv = -1e20;
  static constexpr double logmax = 46.05170185988091;
  static constexpr double c0 = 0.28209479177387814;
  static constexpr double c1 = 0.4886025119029199;
  static constexpr double c2[5] = {1.0925484305920792, -1.0925484305920792, 0.31539156525252005,
                                   -1.0925484305920792, 0.5462742152960396};
  static constexpr double c3[7] = {-0.5900435899266435, 2.890611442640554, -0.4570457994644658,
                                   0.3731763325901154, -0.4570457994644658, 1.445305721320277,
                                   -0.5900435899266435};
};

constexpr float kLogCutoff = 5.54f;  // shaders.slang:17
constexpr int kRound = 16;           // shaders.slang:18 (k-buffer size)
constexpr double kSentinel = 1e9;    // shaders.slang:214

template <class T> inline T fmn(T a, T b) { return std::fmin(a, b); }
template <class T> inline T fmx(T a, T b) { return std::fmax(a, b); }
template <class T> inline T clampv(T v, T lo, T hi) { return fmx(fmn(v, hi), lo); }
template <class T> inline T ffma(T a, T b, T c) { return std::fma(a, b, c); }

// safe_div, safe-math.slang:84-91
template <class T> inline T safe_div(T a, T b) {
  if (std::fabs(b) < K<T>::tiny) return clampv(a / K<T>::tiny, K<T>::minv, K<T>::maxv);
  return clampv(a / b, K<T>::minv, K<T>::maxv);
}
// safe_exp, safe-math.slang:141-144
template <class T> inline T safe_exp(T v) { return std::exp(clampv(v, K<T>::minv, K<T>::logmax)); }
template <class T> inline T sgn(T x) { return x > 0 ? T(1) : (x < 0 ? T(-1) : T(0)); }

// tukey_power_ladder(x, -0.1), safe-math.slang:246-253
template <class T> inline T tukey(T x) {
  const T p = T(-0.1);
  const T pm1 = std::fabs(p - T(1));
  const T xs = std::fabs(x) / fmx(K<T>::tiny, pm1);
  return ((sgn(x) * pm1) / p) * (std::pow(xs + T(1), p) - T(1));
}
// d tukey / dx = sign(x)^2 * (|x|/|p-1| + 1)^(p-1)
template <class T> inline T dtukey(T x) {
  const T p = T(-0.1);
  const T pm1 = std::fabs(p - T(1));
  const T xs = std::fabs(x) / fmx(K<T>::tiny, pm1);
  return sgn(x) * sgn(x) * std::pow(xs + T(1), p - T(1));
}

// rotate_vector(v, q): rotation by the conjugate quaternion, q = (r, x, y, z).
// safe-math.slang:236-244. Fixed operation order, no fma.
template <class T> inline void rotate_vector(const T v[3], const T q[4], T out[3]) {
  const T w = q[0], ux = -q[1], uy = -q[2], uz = -q[3];
  const T tx = T(2) * (uy * v[2] - uz * v[1]);
  const T ty = T(2) * (uz * v[0] - ux * v[2]);
  const T tz = T(2) * (ux * v[1] - uy * v[0]);
  out[0] = (v[0] + w * tx) + (uy * tz - uz * ty);
  out[1] = (v[1] + w * ty) + (uz * tx - ux * tz);
  out[2] = (v[2] + w * tz) + (ux * ty - uy * tx);
}
// VJP of rotate_vector w.r.t. q for cotangent g (accumulates into gq).
template <class T> inline void rotate_vector_vjp_q(const T v[3], const T q[4], const T g[3], T gq[4]) {
  const T w = q[0], u[3] = {-q[1], -q[2], -q[3]};
  // r = v + 2w (u x v) + 2 (u (u.v) - v (u.u))
  const T uxv[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
  const T t[3] = {T(2) * uxv[0], T(2) * uxv[1], T(2) * uxv[2]};
  gq[0] += g[0] * t[0] + g[1] * t[1] + g[2] * t[2];
  const T vxg[3] = {v[1] * g[2] - v[2] * g[1], v[2] * g[0] - v[0] * g[2], v[0] * g[1] - v[1] * g[0]};
  const T uv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
  const T gu = g[0] * u[0] + g[1] * u[1] + g[2] * u[2];
  const T gv = g[0] * v[0] + g[1] * v[1] + g[2] * v[2];
  for (int i = 0; i < 3; ++i) {
    const T du = T(2) * w * vxg[i] + T(2) * (uv * g[i] + gu * v[i] - T(2) * gv * u[i]);
    gq[1 + i] -= du;  // u = -q.yzw
  }
}

// Per-ellipsoid matrix W = diag(1/s) * A(q), A(q) v = rotate_vector(v, q).
// The local (unit-sphere) coordinates of a world point x are W (x - mean):
// this is rotate_vector(x - mean, q) / s of tri-intersect.slang:170-173.
template <class T> inline void prim_matrix(const T q[4], const T s[3], T W[9]) {
  for (int j = 0; j < 3; ++j) {
    T e[3] = {T(0), T(0), T(0)};
    e[j] = T(1);
    T col[3];
    rotate_vector(e, q, col);
    for (int i = 0; i < 3; ++i) W[3 * i + j] = col[i] / s[i];
  }
}

template <class T> struct Hit {
  T t0, t1;
  T ocn[3], rdn[3];
};

// Ray/ellipsoid roots, eliIntersect (tri-intersect.slang:115-131) on local coordinates.
template <class T>
inline bool intersect(const T W[9], const T mu[3], const T o[3], const T d[3], Hit<T>& H) {
  const T v0 = o[0] - mu[0], v1 = o[1] - mu[1], v2 = o[2] - mu[2];
  for (int i = 0; i < 3; ++i) {
    H.ocn[i] = ffma(W[3 * i + 2], v2, ffma(W[3 * i + 1], v1, W[3 * i] * v0));
    H.rdn[i] = ffma(W[3 * i + 2], d[2], ffma(W[3 * i + 1], d[1], W[3 * i] * d[0]));
  }
  const T* oc = H.ocn;
  const T* r = H.rdn;
  const T a = ffma(r[2], r[2], ffma(r[1], r[1], r[0] * r[0]));
  const T bp = -ffma(oc[2], r[2], ffma(oc[1], r[1], oc[0] * r[0]));
  const T ba = bp / a;
  const T l0 = ffma(ba, r[0], oc[0]), l1 = ffma(ba, r[1], oc[1]), l2 = ffma(ba, r[2], oc[2]);
  const T ll = ffma(l2, l2, ffma(l1, l1, l0 * l0));
  const T h = a * (T(1) - ll);
  const T c = ffma(oc[2], oc[2], ffma(oc[1], oc[1], oc[0] * oc[0])) - T(1);
  if (!(h >= T(0))) return false;
  const T sq = std::sqrt(h);
  const T qq = bp > T(0) ? bp + sq : (bp < T(0) ? bp - sq : bp);
  const T ra = c / qq, rb = qq / a;
  H.t0 = fmn(ra, rb);
  H.t1 = fmx(ra, rb);
  return true;
}

// SH basis at direction (x, y, z), sh.slang:48-88, fixed operation order.
template <class T> inline void sh_basis(const T dir[3], int deg, T B[16]) {
  const T x = dir[0], y = dir[1], z = dir[2];
  B[0] = K<T>::c0;
  if (deg < 1) return;
  B[1] = (-K<T>::c1) * y;
  B[2] = K<T>::c1 * z;
  B[3] = (-K<T>::c1) * x;
  if (deg < 2) return;
  const T xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
  B[4] = K<T>::c2[0] * xy;
  B[5] = K<T>::c2[1] * yz;
  B[6] = K<T>::c2[2] * ((T(2) * zz - xx) - yy);
  B[7] = K<T>::c2[3] * xz;
  B[8] = K<T>::c2[4] * (xx - yy);
  if (deg < 3) return;
  B[9] = (K<T>::c3[0] * y) * (T(3) * xx - yy);
  B[10] = (K<T>::c3[1] * xy) * z;
  B[11] = (K<T>::c3[2] * y) * ((T(4) * zz - xx) - yy);
  B[12] = (K<T>::c3[3] * z) * ((T(2) * zz - T(3) * xx) - T(3) * yy);
  B[13] = (K<T>::c3[4] * x) * ((T(4) * zz - xx) - yy);
  B[14] = (K<T>::c3[5] * z) * (xx - yy);
  B[15] = (K<T>::c3[6] * x) * (xx - T(3) * yy);
}

// d B_k / d(x,y,z) (rows k, cols xyz), double only.
template <class T> inline void sh_basis_grad(const T dir[3], int deg, T J[16][3]) {
  const T x = dir[0], y = dir[1], z = dir[2];
  for (int k = 0; k < 16; ++k) J[k][0] = J[k][1] = J[k][2] = 0;
  if (deg < 1) return;
  const T C1 = K<T>::c1;
  J[1][1] = -C1;
  J[2][2] = C1;
  J[3][0] = -C1;
  if (deg < 2) return;
  const T* C2 = K<T>::c2;
  J[4][0] = C2[0] * y; J[4][1] = C2[0] * x;
  J[5][1] = C2[1] * z; J[5][2] = C2[1] * y;
  J[6][0] = -T(2) * C2[2] * x; J[6][1] = -T(2) * C2[2] * y; J[6][2] = T(4) * C2[2] * z;
  J[7][0] = C2[3] * z; J[7][2] = C2[3] * x;
  J[8][0] = T(2) * C2[4] * x; J[8][1] = -T(2) * C2[4] * y;
  if (deg < 3) return;
  const T* C3 = K<T>::c3;
  const T xx = x * x, yy = y * y, zz = z * z;
  J[9][0] = T(6) * C3[0] * x * y; J[9][1] = C3[0] * (3 * xx - 3 * yy);
  J[10][0] = C3[1] * y * z; J[10][1] = C3[1] * x * z; J[10][2] = C3[1] * x * y;
  J[11][0] = -T(2) * C3[2] * x * y; J[11][1] = C3[2] * (4 * zz - xx - 3 * yy); J[11][2] = T(8) * C3[2] * y * z;
  J[12][0] = -T(6) * C3[3] * x * z; J[12][1] = -T(6) * C3[3] * y * z; J[12][2] = C3[3] * (6 * zz - 3 * xx - 3 * yy);
  J[13][0] = C3[4] * (4 * zz - 3 * xx - yy); J[13][1] = -T(2) * C3[4] * x * y; J[13][2] = T(8) * C3[4] * x * z;
  J[14][0] = T(2) * C3[5] * x * z; J[14][1] = -T(2) * C3[5] * y * z; J[14][2] = C3[5] * (xx - yy);
  J[15][0] = C3[6] * (3 * xx - 3 * yy); J[15][1] = -T(6) * C3[6] * x * y;
}

template <class T> struct State {  // SplineState, spline-machine.slang:20-32
  T dist[2] = {0, 0};
  T cum[2] = {0, 0};
  T t = 0;
  T drgb[4] = {0, 0, 0, 0};
  T logT = 0;
  T C[3] = {0, 0, 0};
};

// update(), spline-machine.slang:103-138, fixed operation order.
template <class T> inline State<T> update(const State<T>& s, T t, const T dirac[4]) {
  State<T> n;
  const T dt = fmx(t - s.t, T(0));
  const T area = fmx(s.drgb[0] * dt, T(0));
  T rgb[3];
  for (int i = 0; i < 3; ++i) rgb[i] = safe_div(s.drgb[1 + i], s.drgb[0]);
  n.logT = fmx(area + s.logT, T(0));
  const T w = clampv((T(1) - safe_exp(-area)) * safe_exp(-s.logT), T(0), T(1));
  for (int i = 0; i < 3; ++i) n.C[i] = ffma(w, rgb[i], s.C[i]);
  const T m = tukey(((t + s.t) * T(0.5)) * T(1000));
  const T w2 = T(2) * w;
  n.dist[0] = ffma(w2 * m, s.cum[0], s.dist[0]);
  n.dist[1] = ffma(w2, s.cum[1], s.dist[1]);
  n.cum[0] = s.cum[0] + w;
  n.cum[1] = ffma(w, m, s.cum[1]);
  for (int i = 0; i < 4; ++i) n.drgb[i] = s.drgb[i] + dirac[i];
  n.t = t;
  return n;
}

template <class T> struct Scene {
  int64_t N = 0;
  int Kc = 1;   // SH coefficients stored per ellipsoid (feature stride)
  int deg = 0;  // SH degree evaluated
  std::vector<T> W, mu, sigma, feat;
};

template <class T, class S>
Scene<T> make_scene(int64_t N, int Kc, int deg, const S* mean, const S* scale, const S* quat,
                    const S* density, const S* feat) {
  Scene<T> sc;
  sc.N = N;
  sc.Kc = Kc;
  sc.deg = deg;
  sc.W.resize(9 * N);
  sc.mu.resize(3 * N);
  sc.sigma.resize(N);
  sc.feat.resize((size_t)N * Kc * 3);
  for (int64_t p = 0; p < N; ++p) {
    T q[4] = {T(quat[4 * p]), T(quat[4 * p + 1]), T(quat[4 * p + 2]), T(quat[4 * p + 3])};
    T s[3] = {T(scale[3 * p]), T(scale[3 * p + 1]), T(scale[3 * p + 2])};
    prim_matrix(q, s, &sc.W[9 * p]);
    for (int i = 0; i < 3; ++i) sc.mu[3 * p + i] = T(mean[3 * p + i]);
    sc.sigma[p] = T(density[p]);
  }
  for (size_t i = 0; i < sc.feat.size(); ++i) sc.feat[i] = T(feat[i]);
  return sc;
}

template <class T> struct Ray {
  T o[3], d[3], rd[3];
  T B[16];
};

template <class T> inline Ray<T> make_ray(const T ro[3], const T rd[3], T tmin, int deg) {
  Ray<T> r;
  for (int i = 0; i < 3; ++i) {
    r.rd[i] = rd[i];
    r.o[i] = ffma(tmin, rd[i], ro[i]);  // shaders.slang:179 (origin shifted by the raw direction)
  }
  const T dd = ffma(rd[2], rd[2], ffma(rd[1], rd[1], rd[0] * rd[0]));
  const T nrm = std::sqrt(fmx(dd, K<T>::tiny));  // l2_normalize, safe-math.slang:136-139
  for (int i = 0; i < 3; ++i) r.d[i] = safe_div(rd[i], nrm);
  sh_basis(rd, deg, r.B);  // colour is evaluated along the raw ray direction
  return r;
}

template <class T> inline void prim_colour(const Scene<T>& sc, const Ray<T>& r, int64_t p, T c[3]) {
  const int nb = (sc.deg + 1) * (sc.deg + 1);
  const T* f = &sc.feat[(size_t)p * sc.Kc * 3];
  for (int ch = 0; ch < 3; ++ch) {
    T v = ffma(r.B[0], f[ch], T(0.5));
    for (int k = 1; k < nb; ++k) v = ffma(r.B[k], f[3 * k + ch], v);
    c[ch] = v;
  }
}

template <class T> struct Event {
  T t;
  T t0;  // entry time of the same ellipsoid
  int64_t p;
  int exitbit;  // 0 entry, 1 exit
};

template <class T> struct RayResult {
  State<T> st;
  T last_dirac[4] = {0, 0, 0, 0};
  std::vector<int64_t> ev_p;   // consumed events
  std::vector<int> ev_exit;
  std::vector<T> ev_t;
  State<T> init;
  std::vector<int64_t> members;  // ellipsoids containing the ray start
};

// Full forward of one ray. Reference semantics restated as one pass over the ordered
// candidate events: the reference's 16-event rounds restart from the t of the 16th
// event with a strict '>' (events tied with it are dropped), and an exit beyond tmax
// is only seen in the round that also saw its entry (OptiX drops reported hits > tmax).
template <class T>
RayResult<T> trace_one(const Scene<T>& sc, const Ray<T>& r, T tmax, int max_iters) {
  RayResult<T> res;
  std::vector<Event<T>> ev;
  ev.reserve(64);
  State<T> st;
  for (int64_t p = 0; p < sc.N; ++p) {
    Hit<T> H;
    if (!intersect(&sc.W[9 * p], &sc.mu[3 * p], r.o, r.d, H)) continue;
    if (H.t0 <= T(0) && H.t1 > T(0)) res.members.push_back(p);
    if (H.t0 > T(0) && H.t0 <= tmax) ev.push_back({H.t0, H.t0, p, 0});
    if (H.t1 > T(0)) ev.push_back({H.t1, H.t0, p, 1});
  }
  // initial density: ellipsoids containing the (shifted) ray origin, ascending index
  for (int64_t p : res.members) {
    T c[3];
    prim_colour(sc, r, p, c);
    const T sg = sc.sigma[p];
    st.drgb[0] = st.drgb[0] + sg;
    for (int i = 0; i < 3; ++i) st.drgb[1 + i] = st.drgb[1 + i] + sg * c[i];
  }
  res.init = st;
  std::sort(ev.begin(), ev.end(), [](const Event<T>& a, const Event<T>& b) {
    if (a.t != b.t) return a.t < b.t;
    if (a.p != b.p) return a.p < b.p;
    return a.exitbit < b.exitbit;
  });
  T s16 = T(0);
  int cnt16 = 0;
  int iters = 0;
  if (max_iters > 0) {
    for (const auto& e : ev) {
      if (!(e.t > s16)) continue;
      if ((double)e.t > kSentinel) break;
      if (e.exitbit && e.t > tmax && !(e.t0 > s16 && e.t0 <= tmax)) continue;
      T c[3];
      prim_colour(sc, r, e.p, c);
      const T dh = e.exitbit ? -sc.sigma[e.p] : sc.sigma[e.p];
      const T dirac[4] = {dh, dh * c[0], dh * c[1], dh * c[2]};
      st = update(st, e.t, dirac);
      for (int i = 0; i < 4; ++i) res.last_dirac[i] = dirac[i];
      res.ev_p.push_back(e.p);
      res.ev_exit.push_back(e.exitbit);
      res.ev_t.push_back(e.t);
      ++iters;
      if (++cnt16 == kRound) {
        s16 = e.t;
        cnt16 = 0;
      }
      if (!(st.logT < T(kLogCutoff) && iters < max_iters)) break;
    }
  }
  res.st = st;
  return res;
}

template <class F> void parallel_rays(int64_t R, int nthreads, F fn) {
  if (nthreads <= 1 || R < 2) {
    for (int64_t i = 0; i < R; ++i) fn(i);
    return;
  }
  nthreads = (int)std::min<int64_t>(nthreads, R);
  std::vector<std::thread> th;
  for (int k = 0; k < nthreads; ++k) {
    th.emplace_back([&, k]() {
      for (int64_t i = k; i < R; i += nthreads) fn(i);
    });
  }
  for (auto& t : th) t.join();
}

template <class T> inline void write_state(const State<T>& s, T* out16) {
  out16[0] = s.dist[0]; out16[1] = s.dist[1];
  out16[2] = s.cum[0]; out16[3] = s.cum[1];
  out16[4] = out16[5] = out16[6] = T(0);
  out16[7] = s.t;
  for (int i = 0; i < 4; ++i) out16[8 + i] = s.drgb[i];
  out16[12] = s.logT;
  for (int i = 0; i < 3; ++i) out16[13 + i] = s.C[i];
}

template <class T, class S>
int trace_impl(int64_t N, int Kc, int deg, const S* mean, const S* scale, const S* quat,
               const S* density, const S* feat, int64_t R, const S* rayo, const S* rayd, double tmin,
               double tmax, int max_iters, T* out5, T* state16, T* last_dirac4, int32_t* iters,
               int32_t* events, T* depth, int nthreads) {
  Scene<T> sc = make_scene<T>(N, Kc, deg, mean, scale, quat, density, feat);
  parallel_rays(R, nthreads, [&](int64_t j) {
    const T ro[3] = {T(rayo[3 * j]), T(rayo[3 * j + 1]), T(rayo[3 * j + 2])};
    const T rd[3] = {T(rayd[3 * j]), T(rayd[3 * j + 1]), T(rayd[3 * j + 2])};
    Ray<T> r = make_ray(ro, rd, T(tmin), deg);
    RayResult<T> res = trace_one(sc, r, T(tmax), max_iters);
    const State<T>& s = res.st;
    if (out5) {
      out5[5 * j + 0] = s.C[0];
      out5[5 * j + 1] = s.C[1];
      out5[5 * j + 2] = s.C[2];
      out5[5 * j + 3] = T(1) - std::exp(-s.logT);
      out5[5 * j + 4] = s.dist[0] - s.dist[1];
    }
    if (state16) write_state(s, state16 + 16 * j);
    if (last_dirac4)
      for (int i = 0; i < 4; ++i) last_dirac4[4 * j + i] = res.last_dirac[i];
    const int n = (int)res.ev_p.size();
    if (iters) iters[j] = n;
    if (events)
      for (int i = 0; i < n; ++i)
        events[(int64_t)i * R + j] = (int32_t)(2 * res.ev_p[i] + (res.ev_exit[i] ? 0 : 1));
    if (depth) depth[j] = s.t;
  });
  return 0;
}

// ---------------------------------------------------------------- backward
// FP64: exact analytic gradients along a fixed event sequence, states stored from a
// forward replay. FP32 with inverse_replay: the reference's own scheme
// (backwards_kernel.slang:327-361): states recovered from the final state by
// inverse_update_dual (spline-machine.slang:65-100), in float, as the CUDA kernel does.
// Per-thread gradient accumulator, sparse over ellipsoids (a ray touches few of them):
// one row per touched ellipsoid, W (9), mean (3), density (1), features (3 Kc).
template <class T> struct Grad {
  int stride = 0;
  std::unordered_map<int64_t, size_t> at;
  std::vector<T> data;
  T* row(int64_t p) {
    auto it = at.find(p);
    if (it != at.end()) return &data[it->second];
    const size_t off = data.size();
    data.resize(off + stride, T(0));
    at.emplace(p, off);
    return &data[off];
  }
  const T* find(int64_t p) const {
    auto it = at.find(p);
    return it == at.end() ? nullptr : &data[it->second];
  }
};

// VJP of update() (T), cotangent G of the new state -> cotangent of the old
// state (Gs) and of the control point (Gt, Gdirac). Clamps pass the gradient only
// strictly inside their range.
// inverse_update_dual, spline-machine.slang:65-100 (same operation order as the CUDA kernel).
template <class T> inline State<T> inverse_update(const State<T>& n, const T dirac_new[4], T t_old) {
  State<T> s;
  const T dt = fmx(n.t - t_old, T(0));
  for (int i = 0; i < 4; ++i) s.drgb[i] = n.drgb[i] - dirac_new[i];
  s.t = t_old;
  const T area = fmx(s.drgb[0] * dt, T(0));
  T rgb[3];
  for (int i = 0; i < 3; ++i) rgb[i] = safe_div(s.drgb[1 + i], s.drgb[0]);
  s.logT = fmx(n.logT - area, T(0));
  const T w = clampv((T(1) - safe_exp(-area)) * safe_exp(-s.logT), T(0), T(1));
  for (int i = 0; i < 3; ++i) s.C[i] = n.C[i] - w * rgb[i];
  const T m = tukey(((n.t + s.t) * T(0.5)) * T(1000));
  s.cum[0] = n.cum[0] - w;
  s.cum[1] = n.cum[1] - w * m;
  s.dist[0] = n.dist[0] - T(2) * w * m * s.cum[0];
  s.dist[1] = n.dist[1] - T(2) * w * s.cum[1];
  return s;
}

template <class T>
inline void update_vjp(const State<T>& s, T t, const State<T>& G, State<T>& Gs, T& Gt, T Gdirac[4]) {
  const T dt_raw = t - s.t;
  const T dt = std::fmax(dt_raw, T(0));
  const T area_raw = s.drgb[0] * dt;
  const T area = std::fmax(area_raw, T(0));
  T rgb[3];
  for (int i = 0; i < 3; ++i) rgb[i] = safe_div(s.drgb[1 + i], s.drgb[0]);
  const T ea_in = -area, el_in = -s.logT;
  const T e1 = safe_exp(ea_in), e2 = safe_exp(el_in);
  const T wraw = (T(1) - e1) * e2;
  const T w = clampv(wraw, T(0), T(1));
  const T mid = ((t + s.t) * T(0.5)) * T(1000);
  const T m = tukey(mid);

  Gs = State<T>();
  // pass-through terms
  for (int i = 0; i < 2; ++i) Gs.dist[i] = G.dist[i];
  for (int i = 0; i < 3; ++i) Gs.C[i] = G.C[i];
  for (int i = 0; i < 4; ++i) {
    Gs.drgb[i] = G.drgb[i];
    Gdirac[i] = G.drgb[i];
  }
  Gt = G.t;
  // logT' = max(area + logT, 0)
  T g_area = T(0);
  if (area + s.logT > 0) {
    g_area += G.logT;
    Gs.logT += G.logT;
  }
  // w usage
  T g_w = T(0), g_m = T(0);
  for (int i = 0; i < 3; ++i) g_w += G.C[i] * rgb[i];
  g_w += G.dist[0] * T(2) * m * s.cum[0] + G.dist[1] * T(2) * s.cum[1] + G.cum[0] + G.cum[1] * m;
  g_m += G.dist[0] * T(2) * w * s.cum[0] + G.cum[1] * w;
  Gs.cum[0] = G.cum[0] + G.dist[0] * T(2) * w * m;
  Gs.cum[1] = G.cum[1] + G.dist[1] * T(2) * w;
  // rgb = safe_div(drgb_i, drgb_x), custom backward of safe-math.slang:68-80
  for (int i = 0; i < 3; ++i) {
    const T R = G.C[i] * w;
    const T a = s.drgb[1 + i], b = s.drgb[0];
    const T da = std::fabs(b) < K<T>::tiny ? clampv(R / K<T>::tiny, K<T>::minv, K<T>::maxv)
                                                      : clampv(R / b, K<T>::minv, K<T>::maxv);
    const T b2 = b * b;
    const T db = b2 < K<T>::tiny ? clampv(-a / K<T>::tiny * R, K<T>::minv, K<T>::maxv)
                                           : clampv(-a / b2 * R, K<T>::minv, K<T>::maxv);
    Gs.drgb[1 + i] += da;
    Gs.drgb[0] += db;
  }
  // w = clip((1 - e1) * e2, 0, 1)
  if (wraw > T(0) && wraw < T(1)) {
    const T g_wraw = g_w;
    if (ea_in > K<T>::minv && ea_in < K<T>::logmax) g_area += g_wraw * e2 * e1;  // d(1-e1)/darea = e1
    if (el_in > K<T>::minv && el_in < K<T>::logmax) Gs.logT += -g_wraw * (T(1) - e1) * e2;
  }
  // area = max(drgb_x * dt, 0)
  if (area_raw > T(0)) {
    Gs.drgb[0] += g_area * dt;
    const T g_dt = g_area * s.drgb[0];
    if (dt_raw > T(0)) {
      Gt += g_dt;
      Gs.t -= g_dt;
    }
  }
  // m = tukey(((t + t_s)/2) * 1000)
  const T g_mid = g_m * dtukey(mid) * T(500);
  Gt += g_mid;
  Gs.t += g_mid;
}

struct BwdOut {
  double* dmean;
  double* dscale;
  double* dquat;
  double* ddensity;
  double* dfeat;
  double* drayo;
  double* drayd;
};

template <class T>
int backward_impl(int64_t N, int Kc, int deg, const double* mean, const double* scale,
                  const double* quat, const double* density, const double* feat, int64_t R,
                  const double* rayo, const double* rayd, double tmin, double tmax, int max_iters,
                  const int32_t* events, const int32_t* iters, const double* dout5, BwdOut out,
                  int nthreads, bool inverse_replay) {
  (void)tmax;
  Scene<T> sc = make_scene<T>(N, Kc, deg, mean, scale, quat, density, feat);
  const int nb = (deg + 1) * (deg + 1);
  // per-thread accumulators to stay deterministic per thread; reduced at the end
  nthreads = std::max(1, (int)std::min<int64_t>(nthreads, std::max<int64_t>(R, 1)));
  std::vector<Grad<T>> acc(nthreads);
  for (auto& g : acc) g.stride = 13 + 3 * Kc;
  auto ray_fn = [&](int64_t j, Grad<T>& g) {
    double* gro = out.drayo + 3 * j;
    double* grd = out.drayd + 3 * j;
    for (int i = 0; i < 3; ++i) gro[i] = grd[i] = 0.0;
    const int n = iters[j];
    if (n >= max_iters - 1 || n <= 0) return;  // backwards_kernel.slang:304
    const T ro[3] = {T(rayo[3 * j]), T(rayo[3 * j + 1]), T(rayo[3 * j + 2])};
    const T rd[3] = {T(rayd[3 * j]), T(rayd[3 * j + 1]), T(rayd[3 * j + 2])};
    Ray<T> r = make_ray(ro, rd, T(tmin), deg);
    // initial density (members recomputed in T)
    std::vector<int64_t> members;
    std::vector<T> ts(n);
    std::vector<int64_t> ps(n);
    std::vector<int> ex(n);
    for (int i = 0; i < n; ++i) {
      const int32_t id = events[(int64_t)i * R + j];
      ps[i] = id >> 1;
      ex[i] = (id & 1) ? 0 : 1;
    }
    State<T> st;
    for (int64_t p = 0; p < N; ++p) {
      Hit<T> H;
      if (intersect(&sc.W[9 * p], &sc.mu[3 * p], r.o, r.d, H) && H.t0 <= 0 && H.t1 > 0) members.push_back(p);
    }
    for (int64_t p : members) {
      T c[3];
      prim_colour(sc, r, p, c);
      st.drgb[0] += sc.sigma[p];
      for (int i = 0; i < 3; ++i) st.drgb[1 + i] += sc.sigma[p] * c[i];
    }
    std::vector<State<T>> states(n + 1);
    std::vector<Hit<T>> hits(n);
    std::vector<std::array<T, 4>> diracs(n);
    std::vector<std::array<T, 3>> cols(n);
    states[0] = st;
    for (int i = 0; i < n; ++i) {
      Hit<T> H;
      intersect(&sc.W[9 * ps[i]], &sc.mu[3 * ps[i]], r.o, r.d, H);
      hits[i] = H;
      ts[i] = ex[i] ? H.t1 : H.t0;
      T c[3];
      prim_colour(sc, r, ps[i], c);
      const T dh = ex[i] ? -sc.sigma[ps[i]] : sc.sigma[ps[i]];
      diracs[i] = {dh, dh * c[0], dh * c[1], dh * c[2]};
      cols[i] = {c[0], c[1], c[2]};
      states[i + 1] = update(states[i], ts[i], diracs[i].data());
    }
    if (inverse_replay) {
      // the reference's scheme: only the final state is kept; earlier states are undone
      for (int i = n - 1; i >= 0; --i)
        states[i] = inverse_update(states[i + 1], diracs[i].data(), i > 0 ? ts[i - 1] : T(0));
    }
    const State<T>& fin = states[n];
    State<T> G;
    const double* go = dout5 + 5 * j;
    for (int i = 0; i < 3; ++i) G.C[i] = T(go[i]);
    G.logT = T(go[3]) * std::exp(-fin.logT);  // opacity = 1 - exp(-logT)
    G.dist[0] = T(go[4]);
    G.dist[1] = -T(go[4]);
    T G_o[3] = {0, 0, 0}, G_d[3] = {0, 0, 0}, G_B[16] = {0};
    for (int i = n - 1; i >= 0; --i) {
      State<T> Gs;
      T Gt, Gdirac[4];
      update_vjp(states[i], ts[i], G, Gs, Gt, Gdirac);
      const int64_t p = ps[i];
      const T sg = sc.sigma[p];
      const T sign = ex[i] ? T(-1) : T(1);
      const T dh = sign * sg;
      // dirac = dh * (1, c)
      T g_dh = Gdirac[0];
      for (int ch = 0; ch < 3; ++ch) g_dh += Gdirac[1 + ch] * cols[i][ch];
      g.row(p)[12] += sign * g_dh;
      const T* f = &sc.feat[(size_t)p * Kc * 3];
      T* gf = g.row(p) + 13;
      for (int ch = 0; ch < 3; ++ch) {
        const T gc = dh * Gdirac[1 + ch];
        for (int k = 0; k < nb; ++k) {
          gf[3 * k + ch] += r.B[k] * gc;
          G_B[k] += f[3 * k + ch] * gc;
        }
      }
      // t from the intersection: |ocn + t rdn|^2 = 1
      const Hit<T>& H = hits[i];
      const T t = ts[i];
      // hit point on the unit sphere and d|P|^2/dt / 2, in the cancellation-free form
      // P = l +- (sqrt(h)/a) rdn, P.rdn = +-sqrt(h) (l: closest point of the line to the centre)
      T P[3];
      const T* oc = H.ocn;
      const T* rn = H.rdn;
      const T a_ = ffma(rn[2], rn[2], ffma(rn[1], rn[1], rn[0] * rn[0]));
      const T ba_ = -ffma(oc[2], rn[2], ffma(oc[1], rn[1], oc[0] * rn[0])) / a_;
      T l_[3];
      for (int a = 0; a < 3; ++a) l_[a] = ffma(ba_, rn[a], oc[a]);
      const T ll_ = ffma(l_[2], l_[2], ffma(l_[1], l_[1], l_[0] * l_[0]));
      const T sh = std::sqrt(fmx(a_ * (T(1) - ll_), T(0)));
      const T sgn_ = ex[i] ? T(1) : T(-1);
      for (int a = 0; a < 3; ++a) P[a] = ffma(sgn_ * sh / a_, rn[a], l_[a]);
      const T den = sgn_ * sh;
      if (std::fabs(den) > T(K<T>::tiny)) {
        T g_ocn[3], g_rdn[3];
        for (int a = 0; a < 3; ++a) {
          g_ocn[a] = -Gt * P[a] / den;
          g_rdn[a] = -Gt * t * P[a] / den;
        }
        const T* Wp = &sc.W[9 * p];
        const T v[3] = {r.o[0] - sc.mu[3 * p], r.o[1] - sc.mu[3 * p + 1], r.o[2] - sc.mu[3 * p + 2]};
        T* gr = g.row(p);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) {
            gr[3 * a + b] += g_ocn[a] * v[b] + g_rdn[a] * r.d[b];
            const T wo = Wp[3 * a + b] * g_ocn[a];
            gr[9 + b] -= wo;
            G_o[b] += wo;
            G_d[b] += Wp[3 * a + b] * g_rdn[a];
          }
      }
      G = Gs;
    }
    // initial density members
    for (int64_t p : members) {
      T c[3];
      prim_colour(sc, r, p, c);
      const T sg = sc.sigma[p];
      T g_s = G.drgb[0];
      for (int ch = 0; ch < 3; ++ch) g_s += c[ch] * G.drgb[1 + ch];
      g.row(p)[12] += g_s;
      const T* f = &sc.feat[(size_t)p * Kc * 3];
      T* gf = g.row(p) + 13;
      for (int ch = 0; ch < 3; ++ch) {
        const T gc = sg * G.drgb[1 + ch];
        for (int k = 0; k < nb; ++k) {
          gf[3 * k + ch] += r.B[k] * gc;
          G_B[k] += f[3 * k + ch] * gc;
        }
      }
    }
    // ray: o = ro + tmin * rd; d = rd / |rd|; SH basis of the raw rd
    T J[16][3];
    sh_basis_grad(rd, deg, J);
    T g_rd[3] = {0, 0, 0};
    for (int k = 0; k < nb; ++k)
      for (int a = 0; a < 3; ++a) g_rd[a] += G_B[k] * J[k][a];
    const T nrm = std::sqrt(std::fmax(rd[0] * rd[0] + rd[1] * rd[1] + rd[2] * rd[2], K<T>::tiny));
    const T dG = r.d[0] * G_d[0] + r.d[1] * G_d[1] + r.d[2] * G_d[2];
    for (int a = 0; a < 3; ++a) {
      g_rd[a] += (G_d[a] - r.d[a] * dG) / nrm + T(tmin) * G_o[a];
      gro[a] = G_o[a];
      grd[a] = g_rd[a];
    }
  };
  if (nthreads <= 1) {
    for (int64_t j = 0; j < R; ++j) ray_fn(j, acc[0]);
  } else {
    std::vector<std::thread> th;
    for (int k = 0; k < nthreads; ++k)
      th.emplace_back([&, k]() {
        for (int64_t j = k; j < R; j += nthreads) ray_fn(j, acc[k]);
      });
    for (auto& t : th) t.join();
  }
  // reduce (threads in order) and convert W gradients to scale / quaternion gradients;
  // ellipsoids no ray touched get zero gradients
  std::fill(out.dmean, out.dmean + 3 * N, 0.0);
  std::fill(out.dscale, out.dscale + 3 * N, 0.0);
  std::fill(out.dquat, out.dquat + 4 * N, 0.0);
  std::fill(out.ddensity, out.ddensity + N, 0.0);
  std::fill(out.dfeat, out.dfeat + (size_t)N * Kc * 3, 0.0);
  std::vector<int64_t> touched;
  for (auto& g : acc)
    for (const auto& kv : g.at) touched.push_back(kv.first);
  std::sort(touched.begin(), touched.end());
  touched.erase(std::unique(touched.begin(), touched.end()), touched.end());
  std::vector<const T*> rows(acc.size());
  for (int64_t p : touched) {
    for (size_t k = 0; k < acc.size(); ++k) rows[k] = acc[k].find(p);
    T gW[9] = {0}, gmu[3] = {0}, gs = 0;
    for (const T* gr : rows) {
      if (!gr) continue;
      for (int i = 0; i < 9; ++i) gW[i] += gr[i];
      for (int i = 0; i < 3; ++i) gmu[i] += gr[9 + i];
      gs += gr[12];
    }
    const T q[4] = {T(quat[4 * p]), T(quat[4 * p + 1]), T(quat[4 * p + 2]), T(quat[4 * p + 3])};
    const T s[3] = {T(scale[3 * p]), T(scale[3 * p + 1]), T(scale[3 * p + 2])};
    const T* Wp = &sc.W[9 * p];
    T gscale[3] = {0, 0, 0}, gq[4] = {0, 0, 0, 0};
    for (int i = 0; i < 3; ++i)
      for (int jx = 0; jx < 3; ++jx) gscale[i] -= gW[3 * i + jx] * Wp[3 * i + jx] / s[i];
    for (int jx = 0; jx < 3; ++jx) {
      T e[3] = {0, 0, 0};
      e[jx] = T(1);
      T gcol[3];
      for (int i = 0; i < 3; ++i) gcol[i] = gW[3 * i + jx] / s[i];
      rotate_vector_vjp_q(e, q, gcol, gq);
    }
    for (int i = 0; i < 3; ++i) {
      out.dmean[3 * p + i] = gmu[i];
      out.dscale[3 * p + i] = gscale[i];
    }
    for (int i = 0; i < 4; ++i) out.dquat[4 * p + i] = gq[i];
    out.ddensity[p] = gs;
    for (int i = 0; i < Kc * 3; ++i) {
      T v = 0;
      for (const T* gr : rows)
        if (gr) v += gr[13 + i];
      out.dfeat[(size_t)p * Kc * 3 + i] = v;
    }
  }
  return 0;
}

}  // namespace

extern "C" {

// float32 forward with the exact event specification (bit-exact events / iters).
// events: iteration-major (iter * R + ray), reference ids (2p+1 entry, 2p exit), may be null.
int ora_trace_f32(int64_t N, int Kc, int deg, const float* mean, const float* scale, const float* quat,
                  const float* density, const float* feat, int64_t R, const float* rayo, const float* rayd,
                  float tmin, float tmax, int max_iters, float* out5, float* state16, float* last_dirac4,
                  int32_t* iters, int32_t* events, float* depth, int nthreads) {
  return trace_impl<float, float>(N, Kc, deg, mean, scale, quat, density, feat, R, rayo, rayd, tmin, tmax,
                                  max_iters, out5, state16, last_dirac4, iters, events, depth, nthreads);
}

// float64 forward of the same algorithm (events ordered by their float64 times).
int ora_trace_f64(int64_t N, int Kc, int deg, const double* mean, const double* scale, const double* quat,
                  const double* density, const double* feat, int64_t R, const double* rayo,
                  const double* rayd, double tmin, double tmax, int max_iters, double* out5,
                  double* state16, double* last_dirac4, int32_t* iters, int32_t* events, double* depth,
                  int nthreads) {
  return trace_impl<double, double>(N, Kc, deg, mean, scale, quat, density, feat, R, rayo, rayd, tmin, tmax,
                                    max_iters, out5, state16, last_dirac4, iters, events, depth, nthreads);
}

// float64 analytic backward along a given event sequence (events/iters as returned by
// a forward). Gradients are unclipped; rays with iters >= max_iters-1 get none.
int ora_backward_f64(int64_t N, int Kc, int deg, const double* mean, const double* scale,
                     const double* quat, const double* density, const double* feat, int64_t R,
                     const double* rayo, const double* rayd, double tmin, double tmax, int max_iters,
                     const int32_t* events, const int32_t* iters, const double* dout5, double* dmean,
                     double* dscale, double* dquat, double* ddensity, double* dfeat, double* drayo,
                     double* drayd, int nthreads) {
  BwdOut o{dmean, dscale, dquat, ddensity, dfeat, drayo, drayd};
  return backward_impl<double>(N, Kc, deg, mean, scale, quat, density, feat, R, rayo, rayd, tmin, tmax, max_iters,
                               events, iters, dout5, o, nthreads, false);
}

// float32 backward with the reference's scheme: the final state is undone event by event
// (inverse_update_dual) and every VJP runs in float, as the CUDA kernel does. Inputs and
// outputs are double arrays (values rounded to float inside).
int ora_backward_f32_stored(int64_t N, int Kc, int deg, const double* mean, const double* scale,
                            const double* quat, const double* density, const double* feat, int64_t R,
                            const double* rayo, const double* rayd, double tmin, double tmax, int max_iters,
                            const int32_t* events, const int32_t* iters, const double* dout5, double* dmean,
                            double* dscale, double* dquat, double* ddensity, double* dfeat, double* drayo,
                            double* drayd, int nthreads) {
  BwdOut o{dmean, dscale, dquat, ddensity, dfeat, drayo, drayd};
  return backward_impl<float>(N, Kc, deg, mean, scale, quat, density, feat, R, rayo, rayd, tmin, tmax, max_iters,
                              events, iters, dout5, o, nthreads, false);
}

int ora_backward_f32_replay(int64_t N, int Kc, int deg, const double* mean, const double* scale,
                            const double* quat, const double* density, const double* feat, int64_t R,
                            const double* rayo, const double* rayd, double tmin, double tmax, int max_iters,
                            const int32_t* events, const int32_t* iters, const double* dout5, double* dmean,
                            double* dscale, double* dquat, double* ddensity, double* dfeat, double* drayo,
                            double* drayd, int nthreads) {
  BwdOut o{dmean, dscale, dquat, ddensity, dfeat, drayo, drayd};
  return backward_impl<float>(N, Kc, deg, mean, scale, quat, density, feat, R, rayo, rayd, tmin, tmax, max_iters,
                              events, iters, dout5, o, nthreads, true);
}

// float32 intersection of one ray with one ellipsoid (for known-answer tests).
int ora_intersect_f32(const float* mean, const float* scale, const float* quat, const float* rayo,
                      const float* rayd, float tmin, float* t01) {
  float W[9];
  prim_matrix(quat, scale, W);
  Ray<float> r = make_ray(rayo, rayd, tmin, 0);
  Hit<float> H;
  if (!intersect(W, mean, r.o, r.d, H)) return 0;
  t01[0] = H.t0;
  t01[1] = H.t1;
  return 1;
}

int ora_version(void) { return 1; }

}  // extern "C"
