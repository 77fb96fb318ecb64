// mpm_adjoint.cpp -- TEST INFRASTRUCTURE ONLY: float64 reverse-mode adjoint of
// the MPMEngine substep on the CPU (the "reference gradient").
//
// The reference has no adjoint; this file differentiates, in float64, exactly
// the substep the oracle restates (mpm_p2g.comp:17-87, mpm_grid_update.comp:17-102,
// mpm_g2p.comp:70-272, henckyStress mpm_common.glsl:284-293 with svd3's layout)
// for the setting of the differentiable workload: APIC, ELASTIC (Hencky) with
// per-particle Lame parameters, force table (gravity), wall band boundary, no
// colliders or SDF.  Non-smooth events (15 m/s cap, J reset, world clamp,
// particles leaving the grid interior) are counted and reported: gradients are
// only meaningful when none fire.
//
// Matrices here are mathematical (row, column): B[a][c] is GLSL B[c][a].
// Forward P2G is particle-major; sums differ from the per-node gather only by
// reassociation.  The adjoint of every scatter is a gather and vice versa.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

using M = double[3][3];

inline double bsp(double d) {
  double a = std::abs(d);
  if (a < 0.5) return 0.75 - a * a;
  if (a < 1.5) {
    double t = 1.5 - a;
    return 0.5 * t * t;
  }
  return 0.0;
}
inline double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
inline double bspg(double d) {
  double a = std::abs(d);
  if (a < 0.5) return -2.0 * d;
  if (a < 1.5) return -sgn(d) * (1.5 - a);
  return 0.0;
}
inline double bsph(double d) {
  double a = std::abs(d);
  if (a < 0.5) return -2.0;
  if (a < 1.5) return 1.0;
  return 0.0;
}
inline uint32_t expand(uint32_t v) {
  v = (v | (v << 16u)) & 0x030000FFu;
  v = (v | (v << 8u)) & 0x0300F00Fu;
  v = (v | (v << 4u)) & 0x030C30C3u;
  v = (v | (v << 2u)) & 0x09249249u;
  return v;
}
inline uint32_t morton(int x, int y, int z) { return expand(uint32_t(x)) | (expand(uint32_t(y)) << 1) | (expand(uint32_t(z)) << 2); }

// ---------------------------------------------------------------- svd3 (reference algorithm, float64)
// Returns columns u_m (U[:,m]), v_m, signed sigma, following mpm_common.glsl:213-281.
void svdRef(const M F, M U, double s[3], M V) {
  // A = F^T F (math)
  double A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i][j] = F[0][i] * F[0][j] + F[1][i] * F[1][j] + F[2][i] * F[2][j];
  // Jacobi exactly as the shader indexes its (symmetric) GLSL matrix; the GLSL
  // V[r][p] it updates is rows p of the math matrix whose rows are eigenvectors.
  double W[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};  // W[p][r]: row p = eigenvector p
  for (int iter = 0; iter < 20; ++iter) {
    double a01 = A[0][1], a02 = A[0][2], a12 = A[1][2];
    if (std::max(std::abs(a01), std::max(std::abs(a02), std::abs(a12))) < 1e-8) break;
    int p0, p1;
    double apq;
    if (std::abs(a01) >= std::max(std::abs(a02), std::abs(a12))) { p0 = 0; p1 = 1; apq = a01; }
    else if (std::abs(a02) >= std::abs(a12)) { p0 = 0; p1 = 2; apq = a02; }
    else { p0 = 1; p1 = 2; apq = a12; }
    double app = A[p0][p0], aqq = A[p1][p1];
    double tau = (aqq - app) / (2.0 * apq);
    double t = sgn(tau) / (std::abs(tau) + std::sqrt(1.0 + tau * tau));
    double c = 1.0 / std::sqrt(1.0 + t * t), sn = t * c;
    A[p0][p0] = app - t * apq;
    A[p1][p1] = aqq + t * apq;
    A[p0][p1] = A[p1][p0] = 0.0;
    int r = 3 - p0 - p1;
    double arp = A[r][p0], arq = A[r][p1];
    A[r][p0] = A[p0][r] = c * arp - sn * arq;
    A[r][p1] = A[p1][r] = sn * arp + c * arq;
    for (int q = 0; q < 3; ++q) {
      double vp = W[p0][q], vq = W[p1][q];
      W[p0][q] = c * vp - sn * vq;
      W[p1][q] = sn * vp + c * vq;
    }
  }
  for (int i = 0; i < 3; ++i) s[i] = std::sqrt(std::max(A[i][i], 0.0));
  for (int i = 0; i < 2; ++i)
    for (int j = i + 1; j < 3; ++j)
      if (s[j] > s[i]) {
        std::swap(s[i], s[j]);
        for (int q = 0; q < 3; ++q) std::swap(W[i][q], W[j][q]);
      }
  for (int m = 0; m < 3; ++m)
    for (int q = 0; q < 3; ++q) V[q][m] = W[m][q];
  for (int m = 0; m < 3; ++m) {
    if (s[m] > 1e-8) {
      for (int q = 0; q < 3; ++q) U[q][m] = (F[q][0] * V[0][m] + F[q][1] * V[1][m] + F[q][2] * V[2][m]) / s[m];
    } else {
      for (int q = 0; q < 3; ++q) U[q][m] = (q == m) ? 1.0 : 0.0;
    }
  }
  double det = U[0][0] * (U[1][1] * U[2][2] - U[2][1] * U[1][2]) - U[0][1] * (U[1][0] * U[2][2] - U[2][0] * U[1][2]) +
               U[0][2] * (U[1][0] * U[2][1] - U[2][0] * U[1][1]);
  if (det < 0) {
    for (int q = 0; q < 3; ++q) U[q][2] = -U[q][2];
    s[2] = -s[2];
  }
}

// tau = U^T diag(k) U (math), the shaders' U * diag * transpose(U) with svd3's layout.
void henckyRef(const M F, double mu, double lam, M tau) {
  M U, V;
  double s[3], e[3];
  svdRef(F, U, s, V);
  for (int m = 0; m < 3; ++m) e[m] = std::log(std::max(std::abs(s[m]), 1e-6));
  double tr = e[0] + e[1] + e[2];
  double k[3];
  for (int m = 0; m < 3; ++m) k[m] = lam * tr + 2.0 * mu * e[m];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) tau[i][j] = k[0] * U[0][i] * U[0][j] + k[1] * U[1][i] * U[1][j] + k[2] * U[2][i] * U[2][j];
}

// Adjoint of henckyRef: given sym(tau_bar) adds to Fbar, mubar, lambar.
void henckyRefAdj(const M F, double mu, double lam, const M tbar_in, M Fbar, double& mubar, double& lambar) {
  M U, V;
  double s[3], e[3];
  svdRef(F, U, s, V);
  M tb;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) tb[i][j] = 0.5 * (tbar_in[i][j] + tbar_in[j][i]);
  for (int m = 0; m < 3; ++m) e[m] = std::log(std::max(std::abs(s[m]), 1e-6));
  double tr = e[0] + e[1] + e[2];
  double k[3];
  for (int m = 0; m < 3; ++m) k[m] = lam * tr + 2.0 * mu * e[m];
  M tau;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) tau[i][j] = k[0] * U[0][i] * U[0][j] + k[1] * U[1][i] * U[1][j] + k[2] * U[2][i] * U[2][j];
  // kbar_m = (U tb U^T)_mm
  double kb[3];
  for (int m = 0; m < 3; ++m) {
    double acc = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) acc += U[m][i] * tb[i][j] * U[m][j];
    kb[m] = acc;
  }
  double ksum = kb[0] + kb[1] + kb[2];
  mubar += 2.0 * (kb[0] * e[0] + kb[1] * e[1] + kb[2] * e[2]);
  lambar += ksum * tr;
  // A = tau tb - tb tau (skew)
  M A;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double a = 0;
      for (int q = 0; q < 3; ++q) a += tau[i][q] * tb[q][j] - tb[i][q] * tau[q][j];
      A[i][j] = a;
    }
  M Pb = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int m = 0; m < 3; ++m) {
    const double eb = lam * ksum + 2.0 * mu * kb[m];
    Pb[m][m] = std::abs(s[m]) > 1e-6 ? eb / s[m] : 0.0;
  }
  for (int i = 0; i < 3; ++i)
    for (int j = i + 1; j < 3; ++j) {
      const double den = s[j] * s[j] - s[i] * s[i];
      if (std::abs(den) < 1e-14) continue;
      const double c = 2.0 * A[i][j] / den;
      Pb[i][j] += c * s[j];
      Pb[j][i] += c * s[i];
    }
  // Fbar += U Pb V^T
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double acc = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) acc += U[a][i] * Pb[i][j] * V[b][j];
      Fbar[a][b] += acc;
    }
}

struct Params {
  double dt, h;
  int res[3];
  int cubeRes;
  double g[3];  // summed force acceleration
};

struct State {
  std::vector<double> x, v, B, F, tau;  // x,v: 3/particle; B,F,tau: 9/particle (math row-major)
};

enum : uint32_t { EV_CAP = 1, EV_JRESET = 2, EV_CLAMP = 4, EV_EDGE = 8 };

struct Diff {
  Params P;
  size_t N = 0;
  std::vector<double> mp, Vp, mu, lam;
  uint32_t events = 0;
  // grid scratch
  std::vector<double> gm, gP, gv, gv0;  // mass, momentum(3), velocity after BC(3), capped velocity before forces(3)
  std::vector<double> gcap;             // cap scale 15/|v| where the 15 m/s cap fired, else 1
  std::vector<uint8_t> mask;            // 3 bits: component kept
  std::vector<double> gPb, gmb, gvb;    // adjoints
  size_t nc = 0;

  void init() {
    nc = size_t(P.cubeRes) * P.cubeRes * P.cubeRes;
    gm.assign(nc, 0); gP.assign(3 * nc, 0); gv.assign(3 * nc, 0); gv0.assign(3 * nc, 0); mask.assign(nc, 0); gcap.assign(nc, 1.0);
    gPb.assign(3 * nc, 0); gmb.assign(nc, 0); gvb.assign(3 * nc, 0);
  }

  // stencil of particle p: cell c (unclamped floor == clamped for interior particles)
  bool stencil(const double* x, int c[3]) {
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      double l = x[a] / P.h;
      int f = int(std::floor(l));
      if (f < 1 || f > P.res[a] - 2) ok = false;
      c[a] = std::min(std::max(f, 0), P.res[a] - 1);
    }
    if (!ok) events |= EV_EDGE;
    return ok;
  }

  struct W {
    double w, dw[3], H[3][3], r[3];
  };
  W weight(const double* x, int nx, int ny, int nz) {
    W o;
    const int n[3] = {nx, ny, nz};
    double N[3], Np[3], Npp[3];
    for (int a = 0; a < 3; ++a) {
      double xi = (n[a] + 0.5) * P.h;
      double d = (x[a] - xi) / P.h;
      N[a] = bsp(d); Np[a] = bspg(d); Npp[a] = bsph(d);
      o.r[a] = xi - x[a];
    }
    o.w = N[0] * N[1] * N[2];
    o.dw[0] = Np[0] * N[1] * N[2] / P.h;
    o.dw[1] = N[0] * Np[1] * N[2] / P.h;
    o.dw[2] = N[0] * N[1] * Np[2] / P.h;
    const double h2 = P.h * P.h;
    o.H[0][0] = Npp[0] * N[1] * N[2] / h2; o.H[1][1] = N[0] * Npp[1] * N[2] / h2; o.H[2][2] = N[0] * N[1] * Npp[2] / h2;
    o.H[0][1] = o.H[1][0] = Np[0] * Np[1] * N[2] / h2;
    o.H[0][2] = o.H[2][0] = Np[0] * N[1] * Np[2] / h2;
    o.H[1][2] = o.H[2][1] = N[0] * Np[1] * Np[2] / h2;
    return o;
  }

  void p2g(const State& s) {
    std::fill(gm.begin(), gm.end(), 0.0);
    std::fill(gP.begin(), gP.end(), 0.0);
    const double Dinv = 4.0 / (P.h * P.h);
    for (size_t p = 0; p < N; ++p) {
      const double* x = &s.x[3 * p];
      int c[3];
      stencil(x, c);
      const double* B = &s.B[9 * p];
      const double* T = &s.tau[9 * p];
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int n[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
            if (n[0] < 0 || n[1] < 0 || n[2] < 0 || n[0] >= P.cubeRes || n[1] >= P.cubeRes || n[2] >= P.cubeRes) continue;
            W o = weight(x, n[0], n[1], n[2]);
            if (o.w < 1e-12) continue;
            size_t id = morton(n[0], n[1], n[2]);
            gm[id] += o.w * mp[p];
            for (int a = 0; a < 3; ++a) {
              double Br = B[3 * a] * o.r[0] + B[3 * a + 1] * o.r[1] + B[3 * a + 2] * o.r[2];
              double Td = T[3 * a] * o.dw[0] + T[3 * a + 1] * o.dw[1] + T[3 * a + 2] * o.dw[2];
              gP[3 * id + a] += o.w * mp[p] * (s.v[3 * p + a] + Dinv * Br) - P.dt * Vp[p] * Td;
            }
          }
    }
  }

  void grid() {
    for (size_t id = 0; id < nc; ++id) {
      mask[id] = 0;
      if (gm[id] < 1e-10) continue;
      double v[3];
      for (int a = 0; a < 3; ++a) v[a] = gP[3 * id + a] / gm[id];
      const double speed = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      gcap[id] = 1.0;
      if (speed > 15.0) {
        events |= EV_CAP;
        gcap[id] = 15.0 / speed;
        for (int a = 0; a < 3; ++a) v[a] *= gcap[id];
      }
      int ij[3];
      ij[0] = 0; ij[1] = 0; ij[2] = 0;
      for (int b = 0; b < 10; ++b) {
        ij[0] |= int((id >> (3 * b)) & 1u) << b;
        ij[1] |= int((id >> (3 * b + 1)) & 1u) << b;
        ij[2] |= int((id >> (3 * b + 2)) & 1u) << b;
      }
      uint8_t mk = 0;
      for (int a = 0; a < 3; ++a) {
        gv0[3 * id + a] = v[a];
        double u = v[a] + P.g[a] * P.dt;
        bool zero = (ij[a] <= 1 && u < 0) || (ij[a] >= P.res[a] - 2 && u > 0);
        gv[3 * id + a] = zero ? 0.0 : u;
        if (!zero) mk |= uint8_t(1u << a);
      }
      mask[id] = mk | 8u;  // bit 3: active node
    }
  }

  void g2p(const State& s, State& o) {
    for (size_t p = 0; p < N; ++p) {
      const double* x = &s.x[3 * p];
      int c[3];
      stencil(x, c);
      double vp[3] = {0, 0, 0}, B[9] = {0}, G[9] = {0};
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int n[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
            if (n[0] < 0 || n[1] < 0 || n[2] < 0 || n[0] >= P.res[0] || n[1] >= P.res[1] || n[2] >= P.res[2]) continue;
            size_t id = morton(n[0], n[1], n[2]);
            if (!(mask[id] & 8u)) continue;
            W w = weight(x, n[0], n[1], n[2]);
            if (w.w < 1e-12) continue;
            const double* vi = &gv[3 * id];
            for (int a = 0; a < 3; ++a) {
              vp[a] += w.w * vi[a];
              for (int b = 0; b < 3; ++b) {
                B[3 * a + b] += w.w * vi[a] * w.r[b];
                G[3 * a + b] += vi[a] * w.dw[b];
              }
            }
          }
      const double* F = &s.F[9 * p];
      M Fn, tau;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double acc = F[3 * a + b];
          for (int q = 0; q < 3; ++q) acc += P.dt * G[3 * a + q] * F[3 * q + b];
          Fn[a][b] = acc;
        }
      double J = Fn[0][0] * (Fn[1][1] * Fn[2][2] - Fn[2][1] * Fn[1][2]) - Fn[0][1] * (Fn[1][0] * Fn[2][2] - Fn[2][0] * Fn[1][2]) +
                 Fn[0][2] * (Fn[1][0] * Fn[2][1] - Fn[2][0] * Fn[1][1]);
      if (std::abs(J) < 0.15 || std::abs(J) > 10) events |= EV_JRESET;
      henckyRef(Fn, mu[p], lam[p], tau);
      for (int a = 0; a < 3; ++a) {
        double xn = x[a] + P.dt * vp[a];
        double lo = 1.5 * P.h, hi = P.res[a] * P.h - 1.5 * P.h;
        if (xn < lo || xn > hi) events |= EV_CLAMP;
        o.x[3 * p + a] = xn;
        o.v[3 * p + a] = vp[a];
        for (int b = 0; b < 3; ++b) {
          o.B[9 * p + 3 * a + b] = B[3 * a + b];
          o.F[9 * p + 3 * a + b] = Fn[a][b];
          o.tau[9 * p + 3 * a + b] = tau[a][b];
        }
      }
    }
  }

  void step(const State& s, State& o) {
    p2g(s);
    grid();
    g2p(s, o);
  }

  // Reverse of one substep.  a' (adjoints of outputs) in `ob`; writes adjoints of
  // inputs into `ib` and adds to mu/lam adjoints.  Requires the grid of this
  // substep (p2g + grid run on `s`).
  void stepAdj(const State& s, const State& ob, State& ib, std::vector<double>& mub, std::vector<double>& lamb) {
    std::fill(gvb.begin(), gvb.end(), 0.0);
    const double dt = P.dt;
    const double Dinv = 4.0 / (P.h * P.h);
    // ---- G2P adjoint: per particle, scatter to the grid velocity adjoint
    std::vector<double> Gbar(9 * N), Fkeep(9 * N);
    for (size_t p = 0; p < N; ++p) {
      const double* x = &s.x[3 * p];
      int c[3];
      stencil(x, c);
      // recompute G and F_new
      double G[9] = {0};
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int n[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
            if (n[0] < 0 || n[1] < 0 || n[2] < 0 || n[0] >= P.res[0] || n[1] >= P.res[1] || n[2] >= P.res[2]) continue;
            size_t id = morton(n[0], n[1], n[2]);
            if (!(mask[id] & 8u)) continue;
            W w = weight(x, n[0], n[1], n[2]);
            if (w.w < 1e-12) continue;
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) G[3 * a + b] += gv[3 * id + a] * w.dw[b];
          }
      const double* F = &s.F[9 * p];
      M Fn;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double acc = F[3 * a + b];
          for (int q = 0; q < 3; ++q) acc += dt * G[3 * a + q] * F[3 * q + b];
          Fn[a][b] = acc;
        }
      // tau' = H(F') adjoint
      M Fnb, tb;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          Fnb[a][b] = ob.F[9 * p + 3 * a + b];
          tb[a][b] = ob.tau[9 * p + 3 * a + b];
        }
      double mb = 0, lb = 0;
      henckyRefAdj(Fn, mu[p], lam[p], tb, Fnb, mb, lb);
      mub[p] += mb;
      lamb[p] += lb;
      // x' = x + dt v'
      double xb[3], vb[3];
      for (int a = 0; a < 3; ++a) {
        xb[a] = ob.x[3 * p + a];
        vb[a] = ob.v[3 * p + a] + dt * ob.x[3 * p + a];
      }
      // F' = (I + dt G) F
      double Gb[9];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double fb = Fnb[a][b];  // (I + dt G)^T Fnb
          for (int q = 0; q < 3; ++q) fb += dt * G[3 * q + a] * Fnb[q][b];
          ib.F[9 * p + 3 * a + b] = fb;
          double gb = 0;  // dt Fnb F^T
          for (int q = 0; q < 3; ++q) gb += Fnb[a][q] * F[3 * b + q];
          Gb[3 * a + b] = dt * gb;
        }
      const double* Bb = &ob.B[9 * p];
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int n[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
            if (n[0] < 0 || n[1] < 0 || n[2] < 0 || n[0] >= P.res[0] || n[1] >= P.res[1] || n[2] >= P.res[2]) continue;
            size_t id = morton(n[0], n[1], n[2]);
            if (!(mask[id] & 8u)) continue;
            W w = weight(x, n[0], n[1], n[2]);
            if (w.w < 1e-12) continue;
            const double* vi = &gv[3 * id];
            double viVb = 0, viBbr = 0;
            for (int a = 0; a < 3; ++a) {
              double Bbr = Bb[3 * a] * w.r[0] + Bb[3 * a + 1] * w.r[1] + Bb[3 * a + 2] * w.r[2];
              double Gbdw = Gb[3 * a] * w.dw[0] + Gb[3 * a + 1] * w.dw[1] + Gb[3 * a + 2] * w.dw[2];
              gvb[3 * id + a] += w.w * vb[a] + w.w * Bbr + Gbdw;
              viVb += vi[a] * vb[a];
              viBbr += vi[a] * Bbr;
            }
            for (int b = 0; b < 3; ++b) {
              // v' = sum w v_i ; B' = sum w v_i r^T ; G = sum v_i dw^T
              double BtV = Bb[b] * vi[0] + Bb[3 + b] * vi[1] + Bb[6 + b] * vi[2];  // (Bb^T v_i)_b
              double HGtv = 0;
              for (int q = 0; q < 3; ++q) {
                double GtV = Gb[q] * vi[0] + Gb[3 + q] * vi[1] + Gb[6 + q] * vi[2];  // (Gb^T v_i)_q
                HGtv += w.H[b][q] * GtV;
              }
              xb[b] += w.dw[b] * (viVb + viBbr) - w.w * BtV + HGtv;
            }
          }
      for (int a = 0; a < 3; ++a) {
        ib.x[3 * p + a] = xb[a];
        ib.v[3 * p + a] = 0;  // filled by the P2G adjoint
      }
      for (int q = 0; q < 9; ++q) {
        ib.B[9 * p + q] = 0;
        ib.tau[9 * p + q] = 0;
      }
    }
    // ---- grid adjoint
    std::fill(gPb.begin(), gPb.end(), 0.0);
    std::fill(gmb.begin(), gmb.end(), 0.0);
    for (size_t id = 0; id < nc; ++id) {
      if (!(mask[id] & 8u)) continue;
      // v = mask (cap(P/m) + g dt)
      double vcb[3], v0b[3];
      for (int a = 0; a < 3; ++a) vcb[a] = (mask[id] & (1u << a)) ? gvb[3 * id + a] : 0.0;
      const double sc = gcap[id];
      if (sc < 1.0) {
        // capped: vc = v0 * 15/|v0|;  d vc = (15/|v0|)(I - u u^T) d v0, u = v0/|v0| = vc/15
        double u[3], ud = 0;
        for (int a = 0; a < 3; ++a) {
          u[a] = gv0[3 * id + a] / 15.0;
          ud += u[a] * vcb[a];
        }
        for (int a = 0; a < 3; ++a) v0b[a] = sc * (vcb[a] - u[a] * ud);
      } else {
        for (int a = 0; a < 3; ++a) v0b[a] = vcb[a];
      }
      double mb = 0;
      for (int a = 0; a < 3; ++a) {
        gPb[3 * id + a] = v0b[a] / gm[id];
        mb -= v0b[a] * (gP[3 * id + a] / gm[id]) / gm[id];
      }
      gmb[id] = mb;
    }
    // ---- P2G adjoint: per particle, gather from the grid adjoints
    for (size_t p = 0; p < N; ++p) {
      const double* x = &s.x[3 * p];
      int c[3];
      stencil(x, c);
      const double* B = &s.B[9 * p];
      const double* T = &s.tau[9 * p];
      const double* v = &s.v[3 * p];
      double vb[3] = {0, 0, 0}, Bb[9] = {0}, Tb[9] = {0}, xb[3] = {0, 0, 0};
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int n[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
            if (n[0] < 0 || n[1] < 0 || n[2] < 0 || n[0] >= P.cubeRes || n[1] >= P.cubeRes || n[2] >= P.cubeRes) continue;
            size_t id = morton(n[0], n[1], n[2]);
            W w = weight(x, n[0], n[1], n[2]);
            if (w.w < 1e-12) continue;
            const double* Pb = &gPb[3 * id];
            const double mb = gmb[id];
            // m_i += w m_p
            for (int b = 0; b < 3; ++b) xb[b] += mb * mp[p] * w.dw[b];
            double ve[3];
            for (int a = 0; a < 3; ++a) {
              double Br = B[3 * a] * w.r[0] + B[3 * a + 1] * w.r[1] + B[3 * a + 2] * w.r[2];
              ve[a] = v[a] + Dinv * Br;
            }
            double vePb = ve[0] * Pb[0] + ve[1] * Pb[1] + ve[2] * Pb[2];
            for (int a = 0; a < 3; ++a) {
              vb[a] += w.w * mp[p] * Pb[a];
              for (int b = 0; b < 3; ++b) {
                Bb[3 * a + b] += w.w * mp[p] * Dinv * Pb[a] * w.r[b];
                Tb[3 * a + b] += -dt * Vp[p] * Pb[a] * w.dw[b];
              }
            }
            for (int b = 0; b < 3; ++b) {
              double BtP = B[b] * Pb[0] + B[3 + b] * Pb[1] + B[6 + b] * Pb[2];
              double HTP = 0;
              for (int q = 0; q < 3; ++q) {
                double TP = T[q] * Pb[0] + T[3 + q] * Pb[1] + T[6 + q] * Pb[2];  // (T^T Pb)_q
                HTP += w.H[b][q] * TP;
              }
              xb[b] += w.dw[b] * mp[p] * vePb - w.w * mp[p] * Dinv * BtP - dt * Vp[p] * HTP;
            }
          }
      for (int a = 0; a < 3; ++a) {
        ib.x[3 * p + a] += xb[a];
        ib.v[3 * p + a] = vb[a];
      }
      for (int q = 0; q < 9; ++q) {
        ib.B[9 * p + q] = Bb[q];
        ib.tau[9 * p + q] = Tb[q];
      }
    }
  }
};

void allocState(State& s, size_t n) {
  s.x.assign(3 * n, 0); s.v.assign(3 * n, 0);
  s.B.assign(9 * n, 0); s.F.assign(9 * n, 0); s.tau.assign(9 * n, 0);
}

}  // namespace

extern "C" {

// Reverse-mode gradient of L = |COM(x_T) - target|^2 (COM mass-weighted) with
// respect to the initial velocities and per-particle Lame parameters, through
// `nsub` substeps with checkpoints every `every` substeps and recomputation.
// Inputs (double): x0, v0 (3N), Vp, rho (N), mu, lam (N); F0 = I, B0 = 0, tau0 = 0.
// Outputs: loss, gv0 (3N), gmu, glam (N), xT (3N, may be null), events bitmask.
// params: dt, h, res[3], g[3].
int adj_grad(const double* prm, const int* res, size_t n, const double* x0, const double* v0, const double* Vp, const double* rho,
             const double* mu, const double* lam, const double* target, int nsub, int every, double* loss, double* gv0, double* gmu,
             double* glam, double* xT, uint32_t* events) {
  Diff D;
  D.P.dt = prm[0];
  D.P.h = prm[1];
  for (int a = 0; a < 3; ++a) {
    D.P.res[a] = res[a];
    D.P.g[a] = prm[2 + a];
  }
  int m = std::max(res[0], std::max(res[1], res[2]));
  int c = 1;
  while (c < m) c <<= 1;
  D.P.cubeRes = c;
  D.N = n;
  D.init();
  D.mp.resize(n); D.Vp.assign(Vp, Vp + n); D.mu.assign(mu, mu + n); D.lam.assign(lam, lam + n);
  double M = 0;
  for (size_t p = 0; p < n; ++p) {
    D.mp[p] = rho[p] * Vp[p];
    M += D.mp[p];
  }
  if (every < 1) every = 1;
  State s0;
  allocState(s0, n);
  for (size_t i = 0; i < 3 * n; ++i) { s0.x[i] = x0[i]; s0.v[i] = v0[i]; }
  for (size_t p = 0; p < n; ++p) { s0.F[9 * p] = s0.F[9 * p + 4] = s0.F[9 * p + 8] = 1.0; }
  // forward with checkpoints
  std::vector<State> ck;
  State cur = s0, nxt;
  allocState(nxt, n);
  for (int k = 0; k < nsub; ++k) {
    if (k % every == 0) ck.push_back(cur);
    D.step(cur, nxt);
    std::swap(cur, nxt);
  }
  double com[3] = {0, 0, 0};
  for (size_t p = 0; p < n; ++p)
    for (int a = 0; a < 3; ++a) com[a] += D.mp[p] * cur.x[3 * p + a] / M;
  double L = 0, dL[3];
  for (int a = 0; a < 3; ++a) {
    dL[a] = 2.0 * (com[a] - target[a]);
    L += (com[a] - target[a]) * (com[a] - target[a]);
  }
  *loss = L;
  if (xT) std::memcpy(xT, cur.x.data(), 3 * n * sizeof(double));
  // adjoint of the final state
  State ob, ibuf;
  allocState(ob, n);
  allocState(ibuf, n);
  for (size_t p = 0; p < n; ++p)
    for (int a = 0; a < 3; ++a) ob.x[3 * p + a] = dL[a] * D.mp[p] / M;
  std::vector<double> mub(n, 0.0), lamb(n, 0.0);
  // backward over segments
  for (int seg = int(ck.size()) - 1; seg >= 0; --seg) {
    int k0 = seg * every, k1 = std::min(nsub, k0 + every);
    std::vector<State> st;
    st.push_back(ck[seg]);
    for (int k = k0; k < k1 - 1; ++k) {
      State t;
      allocState(t, n);
      D.step(st.back(), t);
      st.push_back(t);
    }
    for (int k = k1 - 1; k >= k0; --k) {
      const State& s = st[k - k0];
      D.p2g(s);
      D.grid();
      D.stepAdj(s, ob, ibuf, mub, lamb);
      std::swap(ob, ibuf);
    }
  }
  for (size_t i = 0; i < 3 * n; ++i) gv0[i] = ob.v[i];
  for (size_t p = 0; p < n; ++p) {
    gmu[p] = mub[p];
    glam[p] = lamb[p];
  }
  *events = D.events;
  return 0;
}

// Loss only (forward), same setting; for finite differences.
int adj_loss(const double* prm, const int* res, size_t n, const double* x0, const double* v0, const double* Vp, const double* rho,
             const double* mu, const double* lam, const double* target, int nsub, double* loss, uint32_t* events) {
  Diff D;
  D.P.dt = prm[0];
  D.P.h = prm[1];
  for (int a = 0; a < 3; ++a) {
    D.P.res[a] = res[a];
    D.P.g[a] = prm[2 + a];
  }
  int m = std::max(res[0], std::max(res[1], res[2]));
  int c = 1;
  while (c < m) c <<= 1;
  D.P.cubeRes = c;
  D.N = n;
  D.init();
  D.mp.resize(n); D.Vp.assign(Vp, Vp + n); D.mu.assign(mu, mu + n); D.lam.assign(lam, lam + n);
  double M = 0;
  for (size_t p = 0; p < n; ++p) {
    D.mp[p] = rho[p] * Vp[p];
    M += D.mp[p];
  }
  State cur, nxt;
  allocState(cur, n);
  allocState(nxt, n);
  for (size_t i = 0; i < 3 * n; ++i) { cur.x[i] = x0[i]; cur.v[i] = v0[i]; }
  for (size_t p = 0; p < n; ++p) { cur.F[9 * p] = cur.F[9 * p + 4] = cur.F[9 * p + 8] = 1.0; }
  for (int k = 0; k < nsub; ++k) {
    D.step(cur, nxt);
    std::swap(cur, nxt);
  }
  double L = 0;
  for (int a = 0; a < 3; ++a) {
    double com = 0;
    for (size_t p = 0; p < n; ++p) com += D.mp[p] * cur.x[3 * p + a] / M;
    L += (com - target[a]) * (com - target[a]);
  }
  *loss = L;
  *events = D.events;
  return 0;
}

// Hencky (reference layout) and its adjoint for unit tests: F, tau, Fbar, tbar row-major math.
void adj_hencky(const double* F, double mu, double lam, double* tau) {
  M f, t;
  for (int i = 0; i < 9; ++i) f[i / 3][i % 3] = F[i];
  henckyRef(f, mu, lam, t);
  for (int i = 0; i < 9; ++i) tau[i] = t[i / 3][i % 3];
}
void adj_hencky_vjp(const double* F, double mu, double lam, const double* tbar, double* Fbar, double* mubar, double* lambar) {
  M f, tb, fb = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int i = 0; i < 9; ++i) {
    f[i / 3][i % 3] = F[i];
    tb[i / 3][i % 3] = tbar[i];
  }
  double mb = 0, lb = 0;
  henckyRefAdj(f, mu, lam, tb, fb, mb, lb);
  for (int i = 0; i < 9; ++i) Fbar[i] = fb[i / 3][i % 3];
  *mubar = mb;
  *lambar = lb;
}

}  // extern "C"
