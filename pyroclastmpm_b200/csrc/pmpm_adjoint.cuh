// Reverse-mode (adjoint) kernels of the USL step for differentiable
// rollouts: gradients of a loss on particle state with respect to the
// per-particle Drucker-Prager parameters (Young's modulus, friction angle)
// and the initial positions and velocities.  No counterpart in the
// reference.
//
// Forward step k maps the particle state s_k = (x, v, F, sigma, eps_e) to
// s_{k+1}; the backward of step k maps the adjoint of s_{k+1} to the adjoint
// of s_k in three kernels, run after the step's P2G has been recomputed from
// the stored s_k:
//   kadj_g2p   per particle: stress update (Jacobian by forward-mode dual
//              numbers), F update and G2P transposed; node velocity adjoints
//              scattered with atomics; position terms through the weight
//              gradients and Hessians
//   kadj_grid  per node: v = p/m, the boundary conditions and p_nt = p + f dt
//              transposed
//   kadj_p2g   per particle: P2G transposed (a gather over the particle's
//              nodes): velocity, stress, volume (-> F) and position adjoints
// Quadratic B-splines (the configuration this serves); gravity and
// NodeDomain as node conditions; Drucker-Prager and inert materials.
#pragma once

#include <climits>

#include "pmpm_kernels.cuh"

namespace pmpm {

// --------------------------------------------------------------------------
// forward-mode dual numbers
// --------------------------------------------------------------------------

template <int N>
struct Dual {
  float v;
  float d[N];
};

template <int N>
__device__ __forceinline__ Dual<N> dconst(float v) {
  Dual<N> r;
  r.v = v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = 0.0f;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N> &a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = -a.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(float a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a * b.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a * b.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  const float inv = 1.0f / b.v;
  r.v = a.v * inv;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> dsqrt(const Dual<N> &a) {
  Dual<N> r;
  r.v = sqrtf(a.v);
  const float h = r.v > 0.0f ? 0.5f / r.v : 0.0f;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * h;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> dsin(const Dual<N> &a) {
  Dual<N> r;
  r.v = sinf(a.v);
  const float c = cosf(a.v);
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * c;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> dcos(const Dual<N> &a) {
  Dual<N> r;
  r.v = cosf(a.v);
  const float s = -sinf(a.v);
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * s;
  return r;
}

// --------------------------------------------------------------------------
// Drucker-Prager update on dual numbers (same branches as dp_update)
// --------------------------------------------------------------------------

// prm: K, G, eta, eta_bar, kc, p_apex (duals), has_apex (plain).
template <int D, int N>
__device__ void dp_update_dual(const Dual<N> prm[6], bool has_apex, const Dual<N> L[9], float dt, Dual<N> eps[9],
                               const float sref[9], Dual<N> S[9]) {
  const Dual<N> &K = prm[0], &G = prm[1], &eta = prm[2], &eta_bar = prm[3], &kc = prm[4], &p_apex = prm[5];
  Dual<N> deps[9];
  {
    Dual<N> W[9];
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int b = 0; b < D; b++) {
        deps[a * D + b] = (0.5f * dt) * (L[a * D + b] + L[b * D + a]);
        W[a * D + b] = (0.5f * dt) * (L[a * D + b] - L[b * D + a]);
      }
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int b = 0; b < D; b++) {
        Dual<N> acc = dconst<N>(0.0f);
#pragma unroll
        for (int k = 0; k < D; k++) acc = acc - W[a * D + k] * eps[k * D + b] + eps[a * D + k] * W[k * D + b];
        deps[a * D + b] = deps[a * D + b] + acc;
      }
  }
  const float p_ref = (1.0f / 3.0f) * ((sref[0] + sref[4]) + sref[8]);
  float s_ref[9];
#pragma unroll
  for (int k = 0; k < 9; k++) s_ref[k] = sref[k];
  s_ref[0] -= p_ref;
  s_ref[4] -= p_ref;
  s_ref[8] -= p_ref;
  Dual<N> eps_tr[9];
#pragma unroll
  for (int k = 0; k < D * D; k++) eps_tr[k] = eps[k] + deps[k];
  Dual<N> ev = dconst<N>(0.0f);
#pragma unroll
  for (int a = 0; a < D; a++) ev = ev + eps_tr[a * D + a];
  const Dual<N> p_tr = dconst<N>(p_ref) + K * ev;
  Dual<N> s_tr[9];
  Dual<N> ss = dconst<N>(0.0f);
  const Dual<N> two_g = 2.0f * G;
  const Dual<N> third_ev = (1.0f / 3.0f) * ev;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      Dual<N> e = (a < D && b < D) ? eps_tr[a * D + b] : dconst<N>(0.0f);
      if (a == b && !(D < 3 && a == 2)) e = e - third_ev;
      s_tr[3 * a + b] = dconst<N>(s_ref[3 * a + b]) + two_g * e;
      ss = ss + s_tr[3 * a + b] * s_tr[3 * a + b];
    }
  const Dual<N> sqrtJ2 = dsqrt(0.5f * ss);
  const Dual<N> Phi = sqrtJ2 + eta * p_tr - kc;
  if (Phi.v <= 0.0f) {
#pragma unroll
    for (int k = 0; k < 9; k++) S[k] = s_tr[k];
    S[0] = S[0] + p_tr;
    S[4] = S[4] + p_tr;
    S[8] = S[8] + p_tr;
#pragma unroll
    for (int k = 0; k < D * D; k++) eps[k] = eps_tr[k];
    return;
  }
  const Dual<N> dgamma = Phi / (K * eta * eta_bar + G);
  Dual<N> p_next = p_tr - K * eta_bar * dgamma;
  Dual<N> s_next[9];
  const bool apex = has_apex && (sqrtJ2.v - G.v * dgamma.v < 0.0f);
  if (apex) {
    p_next = p_apex;
#pragma unroll
    for (int k = 0; k < 9; k++) s_next[k] = dconst<N>(0.0f);
  } else {
    const Dual<N> scale = dconst<N>(1.0f) - (G * dgamma) / sqrtJ2;
#pragma unroll
    for (int k = 0; k < 9; k++) s_next[k] = scale * s_tr[k];
  }
#pragma unroll
  for (int k = 0; k < 9; k++) S[k] = s_next[k];
  S[0] = S[0] + p_next;
  S[4] = S[4] + p_next;
  S[8] = S[8] + p_next;
  const Dual<N> inv2g = dconst<N>(1.0f) / two_g;
  const Dual<N> dpk = (p_next - dconst<N>(p_ref)) / (3.0f * K);
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) {
      Dual<N> e = (s_next[3 * a + b] - dconst<N>(s_ref[3 * a + b])) * inv2g;
      if (a == b) e = e + dpk;
      eps[a * D + b] = e;
    }
}

// Stored-component maps: stress (3D xx yy zz xy xz yz, 2D xx yy xy zz) and
// elastic strain (3D xx yy zz xy xz yz, 2D xx yy xy) -> full 3x3 / DxD entry.
template <int D>
__device__ __forceinline__ int sig_entry(int k) {
  if (D == 2) {
    const int m[4] = {0, 4, 1, 8};
    return m[k];
  }
  const int m[6] = {0, 4, 8, 1, 2, 5};
  return m[k];
}
template <int D>
__device__ __forceinline__ void eps_entry(int k, int &a, int &b) {
  if (D == 2) {
    const int aa[3] = {0, 1, 0}, bb[3] = {0, 1, 1};
    a = aa[k];
    b = bb[k];
  } else {
    const int aa[6] = {0, 1, 2, 0, 0, 1}, bb[6] = {0, 1, 2, 1, 2, 2};
    a = aa[k];
    b = bb[k];
  }
}

// Vector-Jacobian product of the Drucker-Prager update: inputs L (D*D),
// stored eps (E) and, with per-particle parameters, E and phi; outputs the
// stored stress (S) and stored eps (E).  Input directions are seeded in
// passes of NPASS at a time.
template <int D>
__device__ void dp_vjp(const DevMaterial &mt, bool per_particle, float Ep, float phip, const float L[9], float dt,
                       const float eps_s[6], const float sref[9], const float sbar[6], const float ebar[6],
                       float Lbar[9], float epsbar[6], float &Ebar, float &phibar) {
  constexpr int NS = Sym<D>::S, NE = Sym<D>::E;
  constexpr int NIN = D * D + NE + 2;
  constexpr int NP = 6;
  float gin[NIN];
#pragma unroll
  for (int k = 0; k < NIN; k++) gin[k] = 0.0f;
  for (int base = 0; base < NIN; base += NP) {
    auto seed = [&](int idx, float v) {
      Dual<NP> r = dconst<NP>(v);
      if (idx >= base && idx < base + NP) r.d[idx - base] = 1.0f;
      return r;
    };
    Dual<NP> Ld[9], ed[9], prm[6];
#pragma unroll
    for (int k = 0; k < D * D; k++) Ld[k] = seed(k, L[k]);
#pragma unroll
    for (int k = 0; k < NE; k++) {
      int a, b;
      eps_entry<D>(k, a, b);
      ed[a * D + b] = seed(D * D + k, eps_s[k]);
      if (a != b) ed[b * D + a] = ed[a * D + b];
    }
    bool has_apex;
    if (per_particle) {
      const Dual<NP> E = seed(D * D + NE, Ep);
      const Dual<NP> phi = 0.017453292519943295f * seed(D * D + NE + 1, phip);
      const float nu = mt.p[7], c = mt.p[8];
      const Dual<NP> sn = dsin(phi), cs = dcos(phi);
      const Dual<NP> den = 1.7320508075688772f * (dconst<NP>(3.0f) - sn);
      const Dual<NP> eta = (6.0f * sn) / den, xi = (6.0f * cs) / den;
      prm[0] = (1.0f / (3.0f * (1.0f - 2.0f * nu))) * E;
      prm[1] = (1.0f / (2.0f * (1.0f + nu))) * E;
      prm[2] = eta;
      prm[3] = dconst<NP>(mt.p[3]);
      prm[4] = c * xi;
      prm[5] = eta.v > 0.0f ? prm[4] / eta : dconst<NP>(0.0f);
      has_apex = eta.v > 0.0f;
    } else {
#pragma unroll
      for (int k = 0; k < 6; k++) prm[k] = dconst<NP>(mt.p[k]);
      has_apex = mt.p[6] != 0.0f;
    }
    Dual<NP> S[9];
    dp_update_dual<D, NP>(prm, has_apex, Ld, dt, ed, sref, S);
#pragma unroll
    for (int j = 0; j < NP; j++) {
      if (base + j >= NIN) break;
      float acc = 0.0f;
#pragma unroll
      for (int k = 0; k < NS; k++) acc += sbar[k] * S[sig_entry<D>(k)].d[j];
#pragma unroll
      for (int k = 0; k < NE; k++) {
        int a, b;
        eps_entry<D>(k, a, b);
        acc += ebar[k] * ed[a * D + b].d[j];
      }
      gin[base + j] = acc;
    }
  }
#pragma unroll
  for (int k = 0; k < D * D; k++) Lbar[k] += gin[k];
#pragma unroll
  for (int k = 0; k < NE; k++) epsbar[k] = gin[D * D + k];
  Ebar = gin[D * D + NE];
  phibar = gin[D * D + NE + 1];
}

// Reverse-mode vector-Jacobian product of the Drucker-Prager update (same
// contract as dp_vjp: Lbar accumulates, epsbar / Ebar / phibar are set).
// The primal is recomputed in FP32 with the branch tests of dp_update;
// adjoints follow the forward's expressions in reverse:
//   deps = sym(L) dt - W eps + eps W,  W = skew(L) dt;  eps_tr = eps + deps
//   p_tr = p_ref + K tr(eps_tr);  s_tr = s_ref + 2G dev(eps_tr)  (2D: zz 0)
//   q = sqrt(J2(s_tr));  Phi = q + eta p_tr - kc
//   elastic: S = s_tr + p_tr I, eps' = eps_tr
//   plastic: dgamma = Phi / (K eta eta_bar + G); p = p_tr - K eta_bar dgamma;
//            cone s = (1 - G dgamma / q) s_tr, apex s = 0, p = p_apex;
//            S = s + p I, eps' = (s - s_ref) / 2G + (p - p_ref) / 3K I
template <int D>
__device__ void dp_vjp_rev(const DevMaterial &mt, bool per_particle, float Ep, float phip, const float L[9],
                           float dt, const float eps_s[6], const float sref[9], const float sbar[6],
                           const float ebar[6], float Lbar[9], float epsbar[6], float &Ebar, float &phibar) {
  constexpr int NS = Sym<D>::S, NE = Sym<D>::E;
  // ---- parameters ----
  float K, G, eta, eta_bar, kc, p_apex;
  bool has_apex;
  float nu = 0.0f, c = 0.0f, sn = 0.0f, cs = 0.0f;
  if (per_particle) {
    nu = mt.p[7];
    c = mt.p[8];
    const float phi = phip * 0.017453292519943295f;
    sn = sinf(phi);
    cs = cosf(phi);
    const float den = 1.7320508075688772f * (3.0f - sn);
    eta = 6.0f * sn / den;
    const float xi = 6.0f * cs / den;
    K = Ep / (3.0f * (1.0f - 2.0f * nu));
    G = Ep / (2.0f * (1.0f + nu));
    eta_bar = mt.p[3];
    kc = xi * c;
    p_apex = eta > 0.0f ? kc / eta : 0.0f;
    has_apex = eta > 0.0f;
  } else {
    K = mt.p[0];
    G = mt.p[1];
    eta = mt.p[2];
    eta_bar = mt.p[3];
    kc = mt.p[4];
    p_apex = mt.p[5];
    has_apex = mt.p[6] != 0.0f;
  }
  // ---- primal ----
  float eps[9], Wm[9], deps[9];
#pragma unroll
  for (int k = 0; k < NE; k++) {
    int a, b;
    eps_entry<D>(k, a, b);
    eps[a * D + b] = eps_s[k];
    eps[b * D + a] = eps_s[k];
  }
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) {
      deps[a * D + b] = (0.5f * (L[a * D + b] + L[b * D + a])) * dt;
      Wm[a * D + b] = (0.5f * (L[a * D + b] - L[b * D + a])) * dt;
    }
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) {
      float acc = 0.0f;
#pragma unroll
      for (int k = 0; k < D; k++) acc += -Wm[a * D + k] * eps[k * D + b] + eps[a * D + k] * Wm[k * D + b];
      deps[a * D + b] += acc;
    }
  const float p_ref = (1.0f / 3.0f) * ((sref[0] + sref[4]) + sref[8]);
  float s_ref[9];
#pragma unroll
  for (int k = 0; k < 9; k++) s_ref[k] = sref[k];
  s_ref[0] -= p_ref;
  s_ref[4] -= p_ref;
  s_ref[8] -= p_ref;
  float eps_tr[9];
#pragma unroll
  for (int k = 0; k < D * D; k++) eps_tr[k] = eps[k] + deps[k];
  float ev = 0.0f;
#pragma unroll
  for (int a = 0; a < D; a++) ev += eps_tr[a * D + a];
  const float p_tr = p_ref + K * ev;
  float edev[9], s_tr[9];
  float ss = 0.0f;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      float e = (a < D && b < D) ? eps_tr[a * D + b] : 0.0f;
      if (a == b) e -= (1.0f / 3.0f) * ev;
      if (D < 3 && a == 2 && b == 2) e = 0.0f;
      edev[3 * a + b] = e;
      s_tr[3 * a + b] = s_ref[3 * a + b] + 2.0f * G * e;
      ss += s_tr[3 * a + b] * s_tr[3 * a + b];
    }
  const float q = sqrtf(0.5f * ss);
  const float Phi = (q + eta * p_tr) - kc;
  // ---- output adjoints in full form ----
  float Sb[9], Eb[9];
#pragma unroll
  for (int k = 0; k < 9; k++) Sb[k] = Eb[k] = 0.0f;
#pragma unroll
  for (int k = 0; k < NS; k++) Sb[sig_entry<D>(k)] = sbar[k];
#pragma unroll
  for (int k = 0; k < NE; k++) {
    int a, b;
    eps_entry<D>(k, a, b);
    Eb[a * D + b] = ebar[k];
  }
  float str_b[9], ptr_b = 0.0f, epstr_b[9];
  float Kb = 0.0f, Gb = 0.0f, etab = 0.0f, kcb = 0.0f, papb = 0.0f;
#pragma unroll
  for (int k = 0; k < 9; k++) str_b[k] = epstr_b[k] = 0.0f;
  if (Phi <= 0.0f) {
#pragma unroll
    for (int k = 0; k < 9; k++) str_b[k] = Sb[k];
    ptr_b = Sb[0] + Sb[4] + Sb[8];
#pragma unroll
    for (int k = 0; k < D * D; k++) epstr_b[k] = Eb[k];
  } else {
    const float den = K * eta * eta_bar + G;
    const float dgamma = Phi / den;
    const bool apex = has_apex && (q - G * dgamma < 0.0f);
    float p = p_tr - K * eta_bar * dgamma;
    const float cfac = apex ? 0.0f : 1.0f - G * dgamma / q;
    if (apex) p = p_apex;
    float sv[9];
#pragma unroll
    for (int k = 0; k < 9; k++) sv[k] = cfac * s_tr[k];
    // eps' = (s - s_ref) / 2G + (p - p_ref) / 3K I
    float sb_[9], pb = 0.0f, trEb = 0.0f;
#pragma unroll
    for (int k = 0; k < 9; k++) sb_[k] = Sb[k];
    pb = Sb[0] + Sb[4] + Sb[8];
    const float inv2g = 1.0f / (2.0f * G);
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int b = 0; b < D; b++) {
        const float e = Eb[a * D + b];
        sb_[3 * a + b] += e * inv2g;
        Gb -= e * (sv[3 * a + b] - s_ref[3 * a + b]) * inv2g / G;
      }
#pragma unroll
    for (int a = 0; a < D; a++) trEb += Eb[a * D + a];
    pb += trEb / (3.0f * K);
    Kb -= trEb * (p - p_ref) / (3.0f * K * K);
    float dgb = 0.0f;
    if (apex) {
      papb += pb;
    } else {
      // s = cfac s_tr
      float cb = 0.0f;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        str_b[k] += cfac * sb_[k];
        cb += sb_[k] * s_tr[k];
      }
      // cfac = 1 - G dgamma / q
      Gb -= cb * dgamma / q;
      dgb -= cb * G / q;
      const float qb_c = cb * G * dgamma / (q * q);
      // p = p_tr - K eta_bar dgamma
      ptr_b += pb;
      Kb -= pb * eta_bar * dgamma;
      dgb -= pb * K * eta_bar;
      // q -> s_tr (from cfac)
#pragma unroll
      for (int k = 0; k < 9; k++) str_b[k] += qb_c * s_tr[k] / (2.0f * q);
    }
    // dgamma = Phi / den
    const float Phib = dgb / den;
    const float denb = -dgb * dgamma / den;
    Kb += denb * eta * eta_bar;
    etab += denb * K * eta_bar;
    Gb += denb;
    // Phi = q + eta p_tr - kc
    const float qb = Phib;
    etab += Phib * p_tr;
    ptr_b += Phib * eta;
    kcb -= Phib;
    if (q > 0.0f) {
#pragma unroll
      for (int k = 0; k < 9; k++) str_b[k] += qb * s_tr[k] / (2.0f * q);
    }
  }
  // s_tr = s_ref + 2G edev
  float edev_b[9];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    edev_b[k] = 2.0f * G * str_b[k];
    Gb += 2.0f * str_b[k] * edev[k];
  }
  float evb = 0.0f;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      if (D < 3 && a == 2 && b == 2) continue;
      const float e = edev_b[3 * a + b];
      if (a < D && b < D) epstr_b[a * D + b] += e;
      if (a == b) evb -= (1.0f / 3.0f) * e;
    }
  // p_tr = p_ref + K ev
  evb += K * ptr_b;
  Kb += ev * ptr_b;
#pragma unroll
  for (int a = 0; a < D; a++) epstr_b[a * D + a] += evb;
  // eps_tr = eps + deps; deps = sym dt - W eps + eps W
  float epsb[9], Wb[9];
#pragma unroll
  for (int k = 0; k < D * D; k++) {
    epsb[k] = epstr_b[k];
    Wb[k] = 0.0f;
  }
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++) {
      const float g = epstr_b[a * D + b];
#pragma unroll
      for (int k = 0; k < D; k++) {
        // -W_ak eps_kb
        Wb[a * D + k] -= g * eps[k * D + b];
        epsb[k * D + b] -= g * Wm[a * D + k];
        // eps_ak W_kb
        epsb[a * D + k] += g * Wm[k * D + b];
        Wb[k * D + b] += g * eps[a * D + k];
      }
    }
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int b = 0; b < D; b++)
      Lbar[a * D + b] += 0.5f * dt * (epstr_b[a * D + b] + epstr_b[b * D + a]) +
                         0.5f * dt * (Wb[a * D + b] - Wb[b * D + a]);
#pragma unroll
  for (int k = 0; k < NE; k++) {
    int a, b;
    eps_entry<D>(k, a, b);
    epsbar[k] = a == b ? epsb[a * D + a] : epsb[a * D + b] + epsb[b * D + a];
  }
  Ebar = 0.0f;
  phibar = 0.0f;
  if (per_particle) {
    Ebar = Kb / (3.0f * (1.0f - 2.0f * nu)) + Gb / (2.0f * (1.0f + nu));
    const float s3 = 1.7320508075688772f;
    const float t = 3.0f - sn;
    const float deta = (6.0f / s3) * 3.0f / (t * t) * cs;          // d eta / d phi
    const float dxi = (6.0f / s3) * (1.0f - 3.0f * sn) / (t * t);  // d xi / d phi
    float g = etab * deta + kcb * c * dxi;
    if (eta > 0.0f) g += papb * (c * dxi / eta - kc * deta / (eta * eta));
    phibar = g * 0.017453292519943295f;
  }
}

// --------------------------------------------------------------------------
// quadratic weights with first and second derivatives
// --------------------------------------------------------------------------

// r: relative coordinate in cells; N, dN (per unit length), ddN (per unit length^2).
__device__ __forceinline__ void quad_weight2(float r, float inv_h, float &N, float &dN, float &ddN) {
  const float ar = fabsf(r);
  if (ar < 0.5f) {
    N = 0.75f - r * r;
    dN = inv_h * (-2.0f * r);
    ddN = -2.0f * inv_h * inv_h;
  } else if (ar < 1.5f) {
    const float t = 1.5f - ar;
    N = 0.5f * t * t;
    dN = inv_h * (r > 0.0f ? -t : t);
    ddN = inv_h * inv_h;
  } else {
    N = dN = ddN = 0.0f;
  }
}

// The particle's 3 nodes per axis (boundary-folded indices) with weights.
template <int D>
struct QuadStencil {
  float N[3][3], dN[3][3], ddN[3][3];
  int idx[3][3];
  bool inside;
  __device__ __forceinline__ void build(const DevGrid &g, const float x[3]) {
    inside = true;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int k = 0; k < 3; k++) {
        N[c][k] = 1.0f;
        dN[c][k] = ddN[c][k] = 0.0f;
        idx[c][k] = 0;
      }
#pragma unroll
    for (int c = 0; c < D; c++) {
      const float u = scaled_coord(x[c], g.origin[c], g.inv_h);
      const int b = (int)u;
      inside = inside && b >= 0 && b < g.n[c];
      const int w0 = (u - (float)(b - 1)) < 1.5f ? -1 : 0;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const int sel = b + w0 + k;
        quad_weight2(u - (float)sel, g.inv_h, N[c][k], dN[c][k], ddN[c][k]);
        idx[c][k] = min(max(sel, 0), g.n[c] - 1);
      }
    }
  }
  // weight, gradient and Hessian (row-major DxD) of stencil node (kx, ky, kz)
  __device__ __forceinline__ float eval(int kx, int ky, int kz, float gw[3], float H[9]) const {
    const float nx = N[0][kx], ny = N[1][ky], nz = D == 3 ? N[2][kz] : 1.0f;
    const float dx = dN[0][kx], dy = dN[1][ky], dz = D == 3 ? dN[2][kz] : 0.0f;
    const float hx = ddN[0][kx], hy = ddN[1][ky], hz = D == 3 ? ddN[2][kz] : 0.0f;
    gw[0] = dx * ny * nz;
    gw[1] = nx * dy * nz;
    gw[2] = D == 3 ? nx * ny * dz : 0.0f;
    if (D == 2) {
      H[0] = hx * ny;
      H[1] = dx * dy;
      H[2] = dx * dy;
      H[3] = nx * hy;
    } else {
      H[0] = hx * ny * nz;
      H[1] = dx * dy * nz;
      H[2] = dx * ny * dz;
      H[3] = H[1];
      H[4] = nx * hy * nz;
      H[5] = nx * dy * dz;
      H[6] = H[2];
      H[7] = H[5];
      H[8] = nx * ny * hz;
    }
    return nx * ny * nz;
  }
  __device__ __forceinline__ int node(const DevGrid &g, int kx, int ky, int kz) const {
    return idx[0][kx] + idx[1][ky] * g.n[0] + (D == 3 ? idx[2][kz] * g.n[0] * g.n[1] : 0);
  }
};

// Adjoint state of the particles (SoA by storage slot, stride P.stride) and
// of the nodes (8 floats per node).
struct AdjState {
  float *x, *v, *F, *sig, *eps;  // adjoints of the particle state
  float *gE, *gphi;              // accumulated parameter gradients
  float *node;                   // per node: [0..2] vbar / pbar, [3..5] vntbar / fbar, [6] mbar
  float *Lb;                     // velocity-gradient adjoint between the two G2P backward kernels
};

template <int D>
__device__ __forceinline__ void load_node_vel(const StepArgs &a, int node, float vn[3], float vnt[3]) {
  const float4 *vel = reinterpret_cast<const float4 *>(a.N.vel);
  if (D == 3) {
    const float4 q0 = vel[2 * (size_t)node], q1 = vel[2 * (size_t)node + 1];
    vn[0] = q0.x; vn[1] = q0.y; vn[2] = q0.z;
    vnt[0] = q1.x; vnt[1] = q1.y; vnt[2] = q1.z;
  } else {
    const float4 q = vel[node];
    vn[0] = q.x; vn[1] = q.y; vn[2] = 0.0f;
    vnt[0] = q.z; vnt[1] = q.w; vnt[2] = 0.0f;
  }
}

// Backward of G2P, the F update and the stress update of one particle.
//
// The node adjoints are first summed in shared memory over the node box the
// CTA's particles touch (consecutive storage slots are spatially close: cell
// order after a re-sort, input order otherwise), then added to global
// memory once per node; a CTA whose box exceeds kAdjBoxNodes adds directly.
constexpr int kAdjBoxNodes = 1536;

// First half: the F update and the stress update of one particle.  L is
// recomputed from the step's node velocities; the velocity-gradient adjoint
// goes to A.Lb for the scatter, the F and elastic-strain adjoints are
// replaced in place, the stress adjoint is cleared and the parameter
// gradients are added.  (Split from the scatter so that neither kernel
// carries the other's registers: the return-mapping VJP needs many, the
// scatter its shared-memory node box.)
template <int D>
__global__ void __launch_bounds__(128) kadj_g2p_mat(StepArgs a, AdjState A) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const DevParticles &P = a.P;
  if (s >= P.n) return;
  const DevGrid &g = a.g;
  const int st = P.stride;
  constexpr int NE = Sym<D>::E, NS = Sym<D>::S;
  float x[3] = {0, 0, 0};
#pragma unroll
  for (int c = 0; c < D; c++) x[c] = P.x[c * st + s];
  QuadStencil<D> Q;
  Q.build(g, x);
  float Fb[9], sb[6] = {0, 0, 0, 0, 0, 0}, eb[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < D * D; k++) Fb[k] = A.F[k * st + s];
#pragma unroll
  for (int k = 0; k < NS; k++) sb[k] = A.sig[k * st + s];
#pragma unroll
  for (int k = 0; k < NE; k++) eb[k] = A.eps[k * st + s];
  float Fo[9], eo[6] = {0, 0, 0, 0, 0, 0}, Lb[9];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    Fo[k] = 0.0f;
    Lb[k] = 0.0f;
  }
  if (Q.inside) {
    // recompute L
    float L[9];
#pragma unroll
    for (int k = 0; k < 9; k++) L[k] = 0.0f;
    constexpr int KZ = D == 3 ? 3 : 1;
#pragma unroll
    for (int ky = 0; ky < 3; ky++)
#pragma unroll
      for (int kx = 0; kx < 3; kx++)
#pragma unroll
        for (int kz = 0; kz < KZ; kz++) {
          float gw[3], H[9], vn[3], vnt[3];
          Q.eval(kx, ky, kz, gw, H);
          load_node_vel<D>(a, Q.node(g, kx, ky, kz), vn, vnt);
#pragma unroll
          for (int r = 0; r < D; r++)
#pragma unroll
            for (int c = 0; c < D; c++) L[r * D + c] += gw[r] * vnt[c];
        }
    float F[9];
#pragma unroll
    for (int k = 0; k < D * D; k++) F[k] = P.F[k * st + s];
    // F' = (I + dt L) F: Lbar = dt Fbar' F^T, Fbar = (I + dt L)^T Fbar'
#pragma unroll
    for (int r = 0; r < D; r++)
#pragma unroll
      for (int c = 0; c < D; c++) {
        float acc = 0.0f, accF = 0.0f;
#pragma unroll
        for (int k = 0; k < D; k++) {
          acc += Fb[r * D + k] * F[c * D + k];
          accF += ((k == r ? 1.0f : 0.0f) + a.dt * L[k * D + r]) * Fb[k * D + c];
        }
        Lb[r * D + c] = a.dt * acc;
        Fo[r * D + c] = accF;
      }
    // stress update
    const int color = P.color[s];
    if (color < a.nmat && a.mat[color].type == PMPM_MAT_DRUCKER_PRAGER) {
      const DevMaterial &mt = a.mat[color];
      float eps_s[6] = {0, 0, 0, 0, 0, 0}, sref[9];
#pragma unroll
      for (int k = 0; k < NE; k++) eps_s[k] = P.eps[k * st + s];
      if (a.has_sref) {
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = 0; c < 3; c++) {
            const int k = sig_index<D>(r, c);
            sref[3 * r + c] = k < 0 ? 0.0f : P.sref[k * st + s];
          }
      } else {
#pragma unroll
        for (int k = 0; k < 9; k++) sref[k] = 0.0f;
      }
      const bool pp = P.pE && mt.p[7] >= 0.0f;
      float Ebar = 0.0f, phibar = 0.0f;
      dp_vjp_rev<D>(mt, pp, pp ? P.pE[s] : 0.0f, pp ? P.pphi[s] : 0.0f, L, a.dt, eps_s, sref, sb, eb, Lb, eo, Ebar,
                phibar);
      if (pp) {
        A.gE[s] += Ebar;
        A.gphi[s] += phibar;
      }
    } else {
      // inert material: stress and strain carried through unchanged
#pragma unroll
      for (int k = 0; k < NE; k++) eo[k] = eb[k];
    }
  } else {
    // outside the grid: the particle's state is kept
#pragma unroll
    for (int k = 0; k < D * D; k++) Fo[k] = Fb[k];
#pragma unroll
    for (int k = 0; k < NE; k++) eo[k] = eb[k];
  }
#pragma unroll
  for (int k = 0; k < D * D; k++) {
    A.Lb[k * st + s] = Lb[k];
    A.F[k * st + s] = Fo[k];
  }
#pragma unroll
  for (int k = 0; k < NE; k++) A.eps[k * st + s] = eo[k];
#pragma unroll
  for (int k = 0; k < NS; k++) A.sig[k * st + s] = 0.0f;
}

// Second half: the transposed G2P scatter of one particle (velocity and
// position adjoints; node adjoints summed over the CTA's node box in shared
// memory), with the velocity-gradient adjoint from kadj_g2p_mat.
template <int D>
__global__ void __launch_bounds__(128) kadj_g2p(StepArgs a, AdjState A) {
  __shared__ int box[6];
  __shared__ float acc[kAdjBoxNodes * 6];
  // Storage sorted by cell keeps a cell's particles (8 on a 2x2x2 lattice)
  // together; thread t takes particle (t % 16) * 8 + t / 16 of the CTA's
  // 128, so a warp's lanes spread over 16 cells and their shared-memory
  // atomics on the nodes those cells share collide two ways instead of eight.
  const int s0 = blockIdx.x * 128 + (threadIdx.x & 15) * 8 + (threadIdx.x >> 4);
  const DevParticles &P = a.P;
  const bool valid = s0 < P.n;
  const int s = valid ? s0 : P.n - 1;
  const DevGrid &g = a.g;
  const int st = P.stride;
  float x[3] = {0, 0, 0};
#pragma unroll
  for (int c = 0; c < D; c++) x[c] = P.x[c * st + s];
  QuadStencil<D> Q;
  Q.build(g, x);
  // ---- node box of the CTA ----
  if (threadIdx.x < 3) {
    box[threadIdx.x] = INT_MAX;
    box[3 + threadIdx.x] = -1;
  }
  __syncthreads();
  const bool contributes = valid && Q.inside;
  if (contributes) {
#pragma unroll
    for (int c = 0; c < D; c++) {
      atomicMin(&box[c], Q.idx[c][0]);
      atomicMax(&box[3 + c], Q.idx[c][2]);
    }
  }
  __syncthreads();
  int bx = 1, by = 1, bz = 1, b0x = 0, b0y = 0, b0z = 0;
  if (box[3] >= 0) {
    b0x = box[0];
    b0y = box[1];
    bx = box[3] - box[0] + 1;
    by = box[4] - box[1] + 1;
    if (D == 3) {
      b0z = box[2];
      bz = box[5] - box[2] + 1;
    }
  }
  const bool use_smem = box[3] >= 0 && bx * by * bz <= kAdjBoxNodes;
  const int nbox = use_smem ? bx * by * bz : 0;
  for (int k = threadIdx.x; k < nbox * 6; k += blockDim.x) acc[k] = 0.0f;
  __syncthreads();
  // incoming adjoints (of the step's outputs)
  float xb[3] = {0, 0, 0}, vb[3] = {0, 0, 0};
#pragma unroll
  for (int c = 0; c < D; c++) {
    xb[c] = A.x[c * st + s];
    vb[c] = A.v[c * st + s];
  }
  float xo[3] = {xb[0], xb[1], xb[2]};  // position adjoint: identity part
  float vo[3] = {0, 0, 0};
  if (contributes) {
    float Lb[9];
#pragma unroll
    for (int k = 0; k < D * D; k++) Lb[k] = A.Lb[k * st + s];
    constexpr int KZ = D == 3 ? 3 : 1;
    // G2P transposed
    const float alpha = a.alpha, oma = a.one_minus_alpha;
    float pic[3], dv[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      vo[c] = alpha * vb[c];
      pic[c] = oma * vb[c] + a.dt * xb[c];
      dv[c] = alpha * vb[c];
    }
#pragma unroll
    for (int ky = 0; ky < 3; ky++)
#pragma unroll
      for (int kx = 0; kx < 3; kx++)
#pragma unroll
        for (int kz = 0; kz < KZ; kz++) {
          float gw[3], H[9], vn[3], vnt[3];
          const float w = Q.eval(kx, ky, kz, gw, H);
          const int node = Q.node(g, kx, ky, kz);
          load_node_vel<D>(a, node, vn, vnt);
          float *na;
          if (use_smem) {
            const int lx = Q.idx[0][kx] - b0x, ly = Q.idx[1][ky] - b0y, lz = D == 3 ? Q.idx[2][kz] - b0z : 0;
            na = acc + 6 * (lx + bx * (ly + by * lz));
          } else {
            na = A.node + (size_t)node * 8;
          }
          float coef = 0.0f;  // d/dw of (pic . vnt + dv . (vnt - vn))
#pragma unroll
          for (int c = 0; c < D; c++) {
            float lb = 0.0f;
#pragma unroll
            for (int r = 0; r < D; r++) lb += gw[r] * Lb[r * D + c];
            atomicAdd(na + 3 + c, w * (pic[c] + dv[c]) + lb);
            atomicAdd(na + c, -w * dv[c]);
            coef += pic[c] * vnt[c] + dv[c] * (vnt[c] - vn[c]);
          }
          // position: coef * grad w + Hessian terms of L = sum gw (x) vnt
#pragma unroll
          for (int q = 0; q < D; q++) {
            float hterm = 0.0f;
#pragma unroll
            for (int r = 0; r < D; r++) {
              float lv = 0.0f;
#pragma unroll
              for (int c = 0; c < D; c++) lv += Lb[r * D + c] * vnt[c];
              hterm += H[r * D + q] * lv;
            }
            xo[q] += coef * gw[q] + hterm;
          }
        }
  } else {
    // outside the grid: the particle does not move
#pragma unroll
    for (int c = 0; c < D; c++) vo[c] = vb[c];
  }
  // ---- box sums -> global node adjoints ----
  __syncthreads();
  for (int k = threadIdx.x; k < nbox; k += blockDim.x) {
    const int lx = k % bx, ly = (k / bx) % by, lz = k / (bx * by);
    const int node = (b0x + lx) + (b0y + ly) * g.n[0] + (D == 3 ? (b0z + lz) * g.n[0] * g.n[1] : 0);
    const float *src = acc + 6 * k;
#pragma unroll
    for (int c = 0; c < 6; c++)
      if (src[c] != 0.0f) atomicAdd(A.node + (size_t)node * 8 + c, src[c]);
  }
  if (!valid) return;
#pragma unroll
  for (int c = 0; c < D; c++) {
    A.x[c * st + s] = xo[c];
    A.v[c * st + s] = vo[c];
  }
}

// Backward of the node update for the nodes of the active tiles:
// v = p/m, v_nt = p_nt/m; BCs in reverse list order (NodeDomain clamps pass
// the adjoint where the clamped value is not at the bound, gravity gives
// m a term); p_nt = p + f dt.  Writes pbar, fbar, mbar over the velocity
// adjoints.
template <int D>
__global__ void __launch_bounds__(TileDims<D>::N) kadj_grid(StepArgs a, AdjState A) {
  using T = TileDims<D>;
  const DevGrid &g = a.g;
  const int tile = blockIdx.x;
  if (a.N.tile_epoch[tile] != a.epoch) return;
  const int tx = tile % g.tdim[0], ty = (tile / g.tdim[0]) % g.tdim[1], tz = tile / (g.tdim[0] * g.tdim[1]);
  const int lx = threadIdx.x % T::X, ly = (threadIdx.x / T::X) % T::Y, lz = threadIdx.x / (T::X * T::Y);
  const int nc[3] = {tx * T::X + lx, ty * T::Y + ly, D == 3 ? tz * T::Z + lz : 0};
  if (nc[0] >= g.n[0] || nc[1] >= g.n[1] || nc[2] >= g.n[2]) return;
  const int node = flat_index(g, nc[0], nc[1], nc[2]);
  float *na = A.node + (size_t)node * 8;
  const float m = a.N.m[node];
  float pb[3] = {0, 0, 0}, ptb[3] = {0, 0, 0}, mb = 0.0f;
  if (m > a.cutoff) {
    const int nt = g.ntotal;
    float p[3] = {0, 0, 0}, pnt[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < D; c++) {
      p[c] = a.N.p[c * nt + node];
      pnt[c] = a.N.pnt[c * nt + node];
      const float vbar = na[c], vtbar = na[3 + c];
      pb[c] = vbar / m;
      ptb[c] = vtbar / m;
      mb -= (vbar * p[c] + vtbar * pnt[c]) / (m * m);
    }
    for (int k = a.nbc - 1; k >= 0; k--) {
      const DevBC &bc = a.bc[k];
      if (bc.type == PMPM_BC_NODEDOMAIN) {
        if (!(m > 0.00001f)) continue;
#pragma unroll
        for (int c = 0; c < D; c++) {
          int mode = -1;
          bool lower = false;
          if (nc[c] < 1) {
            mode = bc.i[c];
            lower = true;
          } else if (nc[c] >= g.n[c] - 1) {
            mode = bc.i[3 + c];
          }
          if (mode == 0) {
#pragma unroll
            for (int e = 0; e < D; e++) pb[e] = ptb[e] = 0.0f;
          } else if (mode == 1) {
            // post-clamp value off the bound <=> the clamp was inactive
            if (lower ? !(p[c] > 0.0f) : !(p[c] < 0.0f)) pb[c] = 0.0f;
            if (lower ? !(pnt[c] > 0.0f) : !(pnt[c] < 0.0f)) ptb[c] = 0.0f;
          }
        }
      } else if (bc.type == PMPM_BC_GRAVITY) {
        if (m > 0.000000001f) {
#pragma unroll
          for (int c = 0; c < D; c++) mb += bc.r[c] * a.dt * ptb[c];
        }
      }
    }
    // p_nt = p + f dt
#pragma unroll
    for (int c = 0; c < D; c++) pb[c] += ptb[c];
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    na[c] = pb[c];
    na[3 + c] = ptb[c] * a.dt;  // fbar
  }
  na[6] = mb;
}

// Backward of P2G: gathers the node adjoints of the particle's stencil.
template <int D>
__global__ void __launch_bounds__(128) kadj_p2g(StepArgs a, AdjState A) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const DevParticles &P = a.P;
  if (s >= P.n) return;
  const DevGrid &g = a.g;
  const int st = P.stride;
  constexpr int NS = Sym<D>::S;
  float x[3] = {0, 0, 0}, v[3] = {0, 0, 0};
#pragma unroll
  for (int c = 0; c < D; c++) {
    x[c] = P.x[c * st + s];
    v[c] = P.v[c * st + s];
  }
  QuadStencil<D> Q;
  Q.build(g, x);
  if (!Q.inside) return;
  const float mp = P.m[s], Vp = P.V[s];
  float S[9];
  load_sig3<D>(P, s, S);
  float xo[3] = {0, 0, 0}, vo[3] = {0, 0, 0}, Sb[9], Vb = 0.0f;
#pragma unroll
  for (int k = 0; k < 9; k++) Sb[k] = 0.0f;
  constexpr int KZ = D == 3 ? 3 : 1;
#pragma unroll
  for (int ky = 0; ky < 3; ky++)
#pragma unroll
    for (int kx = 0; kx < 3; kx++)
#pragma unroll
      for (int kz = 0; kz < KZ; kz++) {
        float gw[3], H[9];
        const float w = Q.eval(kx, ky, kz, gw, H);
        const float *na = A.node + (size_t)Q.node(g, kx, ky, kz) * 8;
        float pb[3] = {na[0], na[1], na[2]}, fb[3] = {na[3], na[4], na[5]};
        const float mb = na[6];
        float pv = 0.0f;
#pragma unroll
        for (int c = 0; c < D; c++) {
          vo[c] += w * mp * pb[c];
          pv += pb[c] * v[c];
        }
        // f_a = -V sum_b S_ab gw_b
        float Sg[3] = {0, 0, 0};
#pragma unroll
        for (int r = 0; r < D; r++)
#pragma unroll
          for (int c = 0; c < D; c++) Sg[r] += S[3 * r + c] * gw[c];
#pragma unroll
        for (int r = 0; r < D; r++) {
          Vb -= fb[r] * Sg[r];
#pragma unroll
          for (int c = 0; c < D; c++) Sb[3 * r + c] -= Vp * fb[r] * gw[c];
        }
        // position: m_p (mbar + pbar . v) grad w - V sum_a fbar_a sum_b S_ab H_b.
#pragma unroll
        for (int q = 0; q < D; q++) {
          float h = 0.0f;
#pragma unroll
          for (int r = 0; r < D; r++) {
            float sh = 0.0f;
#pragma unroll
            for (int c = 0; c < D; c++) sh += S[3 * r + c] * H[c * D + q];
            h += fb[r] * sh;
          }
          xo[q] += mp * (mb + pv) * gw[q] - Vp * h;
        }
      }
  // V = det(F) V0: Fbar += Vbar V0 det(F) F^-T = Vbar V0 cof(F)
  float F[9];
#pragma unroll
  for (int k = 0; k < D * D; k++) F[k] = P.F[k * st + s];
  float cof[9];
  if (D == 2) {
    cof[0] = F[3];
    cof[1] = -F[2];
    cof[2] = -F[1];
    cof[3] = F[0];
  } else {
    cof[0] = F[4] * F[8] - F[5] * F[7];
    cof[1] = F[5] * F[6] - F[3] * F[8];
    cof[2] = F[3] * F[7] - F[4] * F[6];
    cof[3] = F[2] * F[7] - F[1] * F[8];
    cof[4] = F[0] * F[8] - F[2] * F[6];
    cof[5] = F[1] * F[6] - F[0] * F[7];
    cof[6] = F[1] * F[5] - F[2] * F[4];
    cof[7] = F[2] * F[3] - F[0] * F[5];
    cof[8] = F[0] * F[4] - F[1] * F[3];
  }
  const float vv0 = Vb * P.V0[s];
#pragma unroll
  for (int c = 0; c < D; c++) {
    A.x[c * st + s] += xo[c];
    A.v[c * st + s] += vo[c];
  }
#pragma unroll
  for (int k = 0; k < D * D; k++) A.F[k * st + s] += vv0 * cof[k];
  // stored stress components: off-diagonal entries appear twice
#pragma unroll
  for (int k = 0; k < NS; k++) {
    const int e = sig_entry<D>(k);
    const int r = e / 3, c = e % 3;
    A.sig[k * st + s] = r == c ? Sb[e] : Sb[3 * r + c] + Sb[3 * c + r];
  }
}

// Vector-Jacobian product of the single-point Drucker-Prager update, by
// reverse mode (method 0) or forward-mode dual numbers (method 1).  Host
// layouts: L, eps, grad_eps_out, grad_L, grad_eps_in [n][D][D]; sref,
// grad_S [n][3][3]; E, phi (may be null), grad_E, grad_phi [n].  Output
// adjoints of the symmetric results count both entries of a pair; the
// symmetric input eps gets one gradient per independent component, written
// to both of its entries.
template <int D>
__global__ void __launch_bounds__(128) k_point_vjp(DevMaterial mt, int n, float dt, const float *L, const float *eps,
                                                   const float *sref, const float *E, const float *phi,
                                                   const float *gS, const float *gE_out, float *gL, float *geps,
                                                   float *gE, float *gphi, int method) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  constexpr int NS = Sym<D>::S, NE = Sym<D>::E;
  float Li[9], es[6] = {0, 0, 0, 0, 0, 0}, sr[9], sb[6] = {0, 0, 0, 0, 0, 0}, eb[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < D * D; k++) Li[k] = L[(size_t)i * D * D + k];
#pragma unroll
  for (int k = 0; k < 9; k++) sr[k] = sref[(size_t)i * 9 + k];
#pragma unroll
  for (int k = 0; k < NE; k++) {
    int a, b;
    eps_entry<D>(k, a, b);
    es[k] = eps[(size_t)i * D * D + a * D + b];
    eb[k] = gE_out[(size_t)i * D * D + a * D + b] + (a != b ? gE_out[(size_t)i * D * D + b * D + a] : 0.0f);
  }
#pragma unroll
  for (int k = 0; k < NS; k++) {
    const int e = sig_entry<D>(k), r = e / 3, c = e % 3;
    sb[k] = gS[(size_t)i * 9 + e] + (r != c ? gS[(size_t)i * 9 + 3 * c + r] : 0.0f);
  }
  const bool pp = E != nullptr && mt.p[7] >= 0.0f;
  float Lb[9], epsb[6], Eb = 0.0f, pb = 0.0f;
#pragma unroll
  for (int k = 0; k < 9; k++) Lb[k] = 0.0f;
  if (method == 0)
    dp_vjp_rev<D>(mt, pp, pp ? E[i] : 0.0f, pp ? phi[i] : 0.0f, Li, dt, es, sr, sb, eb, Lb, epsb, Eb, pb);
  else
    dp_vjp<D>(mt, pp, pp ? E[i] : 0.0f, pp ? phi[i] : 0.0f, Li, dt, es, sr, sb, eb, Lb, epsb, Eb, pb);
#pragma unroll
  for (int k = 0; k < D * D; k++) gL[(size_t)i * D * D + k] = Lb[k];
#pragma unroll
  for (int k = 0; k < NE; k++) {
    int a, b;
    eps_entry<D>(k, a, b);
    geps[(size_t)i * D * D + a * D + b] = epsb[k];
    geps[(size_t)i * D * D + b * D + a] = epsb[k];
  }
  gE[i] = Eb;
  gphi[i] = pb;
}

}  // namespace pmpm
