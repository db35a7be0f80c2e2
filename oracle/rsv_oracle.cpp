// CPU oracle for the ring-Ising structured_adjoint statevector path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product
// path is compared against, and the timed CPU baseline.  Nothing in the
// product (gpu_simulation_b200/, standalone_backend/) links or calls it.
//
// It restates, in plain C++17 + OpenMP, the algorithm of the reference
// repository zzEncounter/GPU_Simulation (paths below are relative to that
// project):
//   * circuit / Hamiltonian definition   ring_ising/models/ising.py:11-44
//   * product-state layer 0              cpp/ising_cuda_rotation_kernels.cu:20-41, 677-710
//   * fused RY.RZ pair update            cpp/ising_cuda_rotation_kernels.cu:43-59
//                                        cpp/ising_cuda_kernels.cu:238-284
//   * ring-CNOT permutation, closed form cpp/ising_cuda_kernels.cu:178-236
//   * ring-CNOT permutation, bit loop    cpp/ising_cuda_dense_kernels.cu:265-284
//   * H psi and the energy partials      cpp/ising_cuda_kernels.cu:313-358
//   * structured adjoint schedule        cpp/ising_cuda_structured_adjoint_modes.inc:108-148, 272-373
//   * per-wire fused backward step       cpp/ising_cuda_statevector_grad_kernels.cu:223-319
//   * gate-level inverse walk            cpp/ising_cuda_gate_level_adjoint_modes.inc:147-260
//                                        cpp/ising_cuda_statevector_grad_kernels.cu:125-221
//
// Reductions are deterministic: amplitudes are summed in fixed blocks of
// ORC_BLOCK entries (sequentially inside a block), and block sums are added in
// block order, so results do not depend on the thread count.
//
// Conventions (pinned by the reference): amplitude index bit w is wire w;
// RY(t) = [[c,-s],[s,c]] with c = cos(t/2), s = sin(t/2);
// RZ(p) = diag(e^{-ip/2}, e^{+ip/2}); per-wire gate U = RZ(p) RY(t); a layer is
// U on every wire, then CNOT(0,1), CNOT(1,2), ..., CNOT(n-1,0);
// H = -sum_i Z_i Z_{i+1 mod n} - h sum_i X_i;
// params flat f64[2 n L], index (layer*n + wire)*2 + {0: theta_RY, 1: phi_RZ}.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cplx = std::complex<double>;
using u64 = std::uint64_t;

constexpr u64 ORC_BLOCK = 4096;

inline int popc(u64 x) { return __builtin_popcountll(x); }

// Closed-form ring-CNOT index map, cpp/ising_cuda_kernels.cu:178-205.
// forward (inverse == false): prefix-XOR of the index with bit 0 replaced by
// the parity of index >> 1.  This is the image P(i) of basis state i.
// inverse: P^{-1}(j) = (j ^ (j << 1)) & mask, with bits 0 and 1 flipped when
// the top bit of j is set.
inline u64 ring_perm_closed(u64 index, int n, bool inverse) {
  const u64 mask = (n >= 64) ? ~u64{0} : ((u64{1} << n) - 1);
  if (!inverse) {
    u64 prefix = index;
    prefix ^= prefix << 1;
    prefix ^= prefix << 2;
    prefix ^= prefix << 4;
    prefix ^= prefix << 8;
    prefix ^= prefix << 16;
    prefix ^= prefix << 32;
    prefix &= mask;
    u64 t = prefix & ~u64{1};
    t |= static_cast<u64>(popc(index >> 1) & 1);
    return t;
  }
  u64 t = (index ^ (index << 1)) & mask;
  if ((index >> (n - 1)) & 1) t ^= 3;
  return t;
}

// Gate-by-gate statement of the same permutation,
// cpp/ising_cuda_dense_kernels.cu:265-284 (CNOT(w, w+1 mod n) applied to the
// basis index for w = 0..n-1; the inverse walks the wires backwards).
inline u64 ring_perm_loop(u64 index, int n, bool inverse) {
  u64 t = index;
  if (!inverse) {
    for (int w = 0; w < n; ++w)
      if ((t >> w) & 1) t ^= u64{1} << ((w + 1) % n);
  } else {
    for (int w = n; w-- > 0;)
      if ((t >> w) & 1) t ^= u64{1} << ((w + 1) % n);
  }
  return t;
}

struct Coeffs {
  double c, s, ch, sh;  // cos(theta/2), sin(theta/2), cos(phi/2), sin(phi/2)
};

// Host cos/sin exactly as cpp/ising_cuda_rotation_kernels.cu:661-675.
inline Coeffs make_coeffs(double theta, double phi) {
  const double ry = theta * 0.5;
  const double rz = phi * 0.5;
  return {std::cos(ry), std::sin(ry), std::cos(rz), std::sin(rz)};
}

// Fused RY then RZ on one pair, cpp/ising_cuda_rotation_kernels.cu:43-59.
inline void ryrz_forward_pair(const Coeffs &k, cplx &a0, cplx &a1) {
  const double b0r = k.c * a0.real() - k.s * a1.real();
  const double b0i = k.c * a0.imag() - k.s * a1.imag();
  const double b1r = k.s * a0.real() + k.c * a1.real();
  const double b1i = k.s * a0.imag() + k.c * a1.imag();
  a0 = cplx(k.ch * b0r + k.sh * b0i, k.ch * b0i - k.sh * b0r);
  a1 = cplx(k.ch * b1r - k.sh * b1i, k.ch * b1i + k.sh * b1r);
}

inline u64 pair_base(u64 pair_index, int wire) {
  const u64 low = (u64{1} << wire) - 1;
  return ((pair_index >> wire) << (wire + 1)) | (pair_index & low);
}

void apply_ryrz(cplx *st, int n, int wire, const Coeffs &k) {
  const long long pairs = static_cast<long long>((u64{1} << n) / 2);
#pragma omp parallel for schedule(static)
  for (long long p = 0; p < pairs; ++p) {
    const u64 i0 = pair_base(static_cast<u64>(p), wire);
    const u64 i1 = i0 | (u64{1} << wire);
    ryrz_forward_pair(k, st[i0], st[i1]);
  }
}

// Layer-0 product state, cpp/ising_cuda_rotation_kernels.cu:20-41, 677-710.
void init_product_state(cplx *st, int n, const double *layer_params) {
  std::vector<double> zr(n), zi(n), or_(n), oi(n);
  for (int w = 0; w < n; ++w) {
    const Coeffs k = make_coeffs(layer_params[2 * w], layer_params[2 * w + 1]);
    zr[w] = k.c * k.ch;
    zi[w] = -k.c * k.sh;
    or_[w] = k.s * k.ch;
    oi[w] = k.s * k.sh;
  }
  const long long S = static_cast<long long>(u64{1} << n);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < S; ++i) {
    double vr = 1.0, vi = 0.0;
    for (int w = 0; w < n; ++w) {
      const bool one = (static_cast<u64>(i) >> w) & 1;
      const double fr = one ? or_[w] : zr[w];
      const double fi = one ? oi[w] : zi[w];
      const double nr = vr * fr - vi * fi;
      const double ni = vr * fi + vi * fr;
      vr = nr;
      vi = ni;
    }
    st[i] = cplx(vr, vi);
  }
}

// out[P(i)] = in[i]  (forward ring layer, cpp/ising_cuda_kernels.cu:207-220)
void ring_scatter(cplx *out, const cplx *in, int n) {
  const long long S = static_cast<long long>(u64{1} << n);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < S; ++i)
    out[ring_perm_closed(static_cast<u64>(i), n, false)] = in[i];
}

// out[i] = in[P(i)]  (inverse ring layer, cpp/ising_cuda_kernels.cu:222-236,
// selected with inverse=true by launch_apply_ring_cnot_layer :409-424)
void ring_gather_inverse(cplx *out, const cplx *in, int n) {
  const long long S = static_cast<long long>(u64{1} << n);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < S; ++i)
    out[i] = in[ring_perm_closed(static_cast<u64>(i), n, false)];
}

inline double hamiltonian_diag(u64 i, int n) {
  const u64 mask = (u64{1} << n) - 1;
  const u64 rot = ((i << 1) & mask) | (i >> (n - 1));
  return static_cast<double>(2 * popc((i ^ rot) & mask)) - static_cast<double>(n);
}

// lambda = H psi and E = sum Re(conj(psi) lambda); cpp/ising_cuda_kernels.cu:313-358.
double apply_hamiltonian_energy(cplx *lam, const cplx *st, int n, double field) {
  const u64 S = u64{1} << n;
  const u64 nblocks = (S + ORC_BLOCK - 1) / ORC_BLOCK;
  std::vector<double> part(nblocks, 0.0);
#pragma omp parallel for schedule(static)
  for (long long b = 0; b < static_cast<long long>(nblocks); ++b) {
    double acc = 0.0;
    const u64 lo = static_cast<u64>(b) * ORC_BLOCK;
    const u64 hi = std::min(S, lo + ORC_BLOCK);
    for (u64 i = lo; i < hi; ++i) {
      const cplx a = st[i];
      cplx v = hamiltonian_diag(i, n) * a;
      for (int w = 0; w < n; ++w) v += cplx(-field, 0.0) * st[i ^ (u64{1} << w)];
      lam[i] = v;
      acc += a.real() * v.real() + a.imag() * v.imag();
    }
    part[b] = acc;
  }
  double e = 0.0;
  for (double p : part) e += p;
  return e;
}

// One per-wire fused backward step, cpp/ising_cuda_statevector_grad_kernels.cu:223-319.
// Undoes RZ then RY on psi and lambda in place and returns the theta and phi
// gradient contributions (already multiplied by 2, as the kernel does).
void ryrz_backward_wire(cplx *cur, cplx *lam, int n, int wire, const Coeffs &k,
                        double *gtheta, double *gphi) {
  const u64 pairs = (u64{1} << n) / 2;
  const u64 nblocks = (pairs + ORC_BLOCK - 1) / ORC_BLOCK;
  std::vector<double> pt(nblocks, 0.0), pp(nblocks, 0.0);
#pragma omp parallel for schedule(static)
  for (long long b = 0; b < static_cast<long long>(nblocks); ++b) {
    double ts = 0.0, ps = 0.0;
    const u64 lo = static_cast<u64>(b) * ORC_BLOCK;
    const u64 hi = std::min(pairs, lo + ORC_BLOCK);
    for (u64 p = lo; p < hi; ++p) {
      const u64 i0 = pair_base(p, wire);
      const u64 i1 = i0 | (u64{1} << wire);
      const double ca0r = cur[i0].real(), ca0i = cur[i0].imag();
      const double ca1r = cur[i1].real(), ca1i = cur[i1].imag();
      const double la0r = lam[i0].real(), la0i = lam[i0].imag();
      const double la1r = lam[i1].real(), la1i = lam[i1].imag();
      const double rz_c = k.ch, rz_s = k.sh;
      const double cm0r = rz_c * ca0r - rz_s * ca0i;
      const double cm0i = rz_c * ca0i + rz_s * ca0r;
      const double cm1r = rz_c * ca1r + rz_s * ca1i;
      const double cm1i = rz_c * ca1i - rz_s * ca1r;
      const double lm0r = rz_c * la0r - rz_s * la0i;
      const double lm0i = rz_c * la0i + rz_s * la0r;
      const double lm1r = rz_c * la1r + rz_s * la1i;
      const double lm1i = rz_c * la1i - rz_s * la1r;
      ps += 0.5 * ((la0r * ca0i - la0i * ca0r) - (la1r * ca1i - la1i * ca1r));
      const double ry_c = k.c, ry_s = k.s;
      const double cb0r = ry_c * cm0r + ry_s * cm1r;
      const double cb0i = ry_c * cm0i + ry_s * cm1i;
      const double cb1r = -ry_s * cm0r + ry_c * cm1r;
      const double cb1i = -ry_s * cm0i + ry_c * cm1i;
      cur[i0] = cplx(cb0r, cb0i);
      cur[i1] = cplx(cb1r, cb1i);
      const double d0r = -0.5 * (ry_s * cb0r + ry_c * cb1r);
      const double d0i = -0.5 * (ry_s * cb0i + ry_c * cb1i);
      const double d1r = 0.5 * (ry_c * cb0r - ry_s * cb1r);
      const double d1i = 0.5 * (ry_c * cb0i - ry_s * cb1i);
      ts += lm0r * d0r + lm0i * d0i + lm1r * d1r + lm1i * d1i;
      lam[i0] = cplx(ry_c * lm0r + ry_s * lm1r, ry_c * lm0i + ry_s * lm1i);
      lam[i1] = cplx(-ry_s * lm0r + ry_c * lm1r, -ry_s * lm0i + ry_c * lm1i);
    }
    pt[b] = ts;
    pp[b] = ps;
  }
  double t = 0.0, q = 0.0;
  for (u64 b = 0; b < nblocks; ++b) {
    t += pt[b];
    q += pp[b];
  }
  *gtheta += 2.0 * t;
  *gphi += 2.0 * q;
}

// ---- gate-level pieces (PennyLane gate order: RY, RZ per wire, then CNOTs) ----

void apply_ry(cplx *st, int n, int wire, double theta, bool inverse) {
  const double c = std::cos(theta * 0.5);
  const double s = inverse ? -std::sin(theta * 0.5) : std::sin(theta * 0.5);
  const long long pairs = static_cast<long long>((u64{1} << n) / 2);
#pragma omp parallel for schedule(static)
  for (long long p = 0; p < pairs; ++p) {
    const u64 i0 = pair_base(static_cast<u64>(p), wire);
    const u64 i1 = i0 | (u64{1} << wire);
    const cplx a0 = st[i0], a1 = st[i1];
    st[i0] = c * a0 - s * a1;
    st[i1] = s * a0 + c * a1;
  }
}

void apply_rz(cplx *st, int n, int wire, double phi, bool inverse) {
  const double h = (inverse ? -phi : phi) * 0.5;
  const cplx f0(std::cos(-h), std::sin(-h)), f1(std::cos(h), std::sin(h));
  const long long S = static_cast<long long>(u64{1} << n);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < S; ++i)
    st[i] *= ((static_cast<u64>(i) >> wire) & 1) ? f1 : f0;
}

void apply_cnot(cplx *st, int n, int control, int target) {
  const long long S = static_cast<long long>(u64{1} << n);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < S; ++i) {
    const u64 u = static_cast<u64>(i);
    if (((u >> control) & 1) && !((u >> target) & 1))
      std::swap(st[u], st[u | (u64{1} << target)]);
  }
}

// 2 Re <lam | dRY/dtheta | psi_before>, psi = RY psi_before (grad_kernels.cu:125-178).
double ry_gradient(const cplx *cur, const cplx *lam, int n, int wire, double theta) {
  const double c = std::cos(theta * 0.5), s = std::sin(theta * 0.5);
  const u64 pairs = (u64{1} << n) / 2;
  const u64 nblocks = (pairs + ORC_BLOCK - 1) / ORC_BLOCK;
  std::vector<double> part(nblocks, 0.0);
#pragma omp parallel for schedule(static)
  for (long long b = 0; b < static_cast<long long>(nblocks); ++b) {
    double acc = 0.0;
    const u64 lo = static_cast<u64>(b) * ORC_BLOCK;
    const u64 hi = std::min(pairs, lo + ORC_BLOCK);
    for (u64 p = lo; p < hi; ++p) {
      const u64 i0 = pair_base(p, wire);
      const u64 i1 = i0 | (u64{1} << wire);
      const cplx b0 = c * cur[i0] + s * cur[i1];
      const cplx b1 = -s * cur[i0] + c * cur[i1];
      const cplx d0 = (-0.5 * s) * b0 + (-0.5 * c) * b1;
      const cplx d1 = (0.5 * c) * b0 + (-0.5 * s) * b1;
      acc += (std::conj(lam[i0]) * d0 + std::conj(lam[i1]) * d1).real();
    }
    part[b] = acc;
  }
  double t = 0.0;
  for (double p : part) t += p;
  return 2.0 * t;
}

// 2 Re <lam | dRZ/dphi | psi_before> (grad_kernels.cu:180-221).
double rz_gradient(const cplx *cur, const cplx *lam, int n, int wire, double phi) {
  const u64 S = u64{1} << n;
  const u64 nblocks = (S + ORC_BLOCK - 1) / ORC_BLOCK;
  std::vector<double> part(nblocks, 0.0);
  const double h = phi * 0.5;
#pragma omp parallel for schedule(static)
  for (long long b = 0; b < static_cast<long long>(nblocks); ++b) {
    double acc = 0.0;
    const u64 lo = static_cast<u64>(b) * ORC_BLOCK;
    const u64 hi = std::min(S, lo + ORC_BLOCK);
    for (u64 i = lo; i < hi; ++i) {
      const bool bit = (i >> wire) & 1;
      const double fph = bit ? h : -h;
      const cplx fwd(std::cos(fph), std::sin(fph));
      const cplx inv(std::cos(-fph), std::sin(-fph));
      const cplx pre = bit ? cplx(0.0, 0.5) : cplx(0.0, -0.5);
      acc += (std::conj(lam[i]) * pre * fwd * (inv * cur[i])).real();
    }
    part[b] = acc;
  }
  double t = 0.0;
  for (double p : part) t += p;
  return 2.0 * t;
}

int orc_threads = 0;

void set_threads() {
#ifdef _OPENMP
  if (orc_threads > 0) omp_set_num_threads(orc_threads);
#endif
}

bool valid_shape(int n, int L) { return n >= 2 && n <= 34 && L >= 1; }

// structured_adjoint forward: cpp/ising_cuda_structured_adjoint_modes.inc:108-148.
// On return cur holds the final state; scratch is clobbered.
void structured_forward(std::vector<cplx> &cur, std::vector<cplx> &scratch, int n, int L,
                        const double *params) {
  init_product_state(cur.data(), n, params);
  ring_scatter(scratch.data(), cur.data(), n);
  std::swap(cur, scratch);
  for (int layer = 1; layer < L; ++layer) {
    for (int w = 0; w < n; ++w) {
      const double *p = params + 2 * (static_cast<std::size_t>(layer) * n + w);
      apply_ryrz(cur.data(), n, w, make_coeffs(p[0], p[1]));
    }
    ring_scatter(scratch.data(), cur.data(), n);
    std::swap(cur, scratch);
  }
}

void gate_level_forward(std::vector<cplx> &cur, int n, int L, const double *params) {
  std::fill(cur.begin(), cur.end(), cplx(0.0, 0.0));
  cur[0] = 1.0;
  for (int layer = 0; layer < L; ++layer) {
    for (int w = 0; w < n; ++w) {
      const double *p = params + 2 * (static_cast<std::size_t>(layer) * n + w);
      apply_ry(cur.data(), n, w, p[0], false);
      apply_rz(cur.data(), n, w, p[1], false);
    }
    for (int w = 0; w < n; ++w) apply_cnot(cur.data(), n, w, (w + 1) % n);
  }
}

}  // namespace

extern "C" {

// Thread count used by the oracle (0 = OpenMP default = all host threads).
void orc_set_num_threads(int k) { orc_threads = k; }

int orc_get_num_threads() {
#ifdef _OPENMP
  set_threads();
  int t = 1;
#pragma omp parallel
  {
#pragma omp single
    t = omp_get_num_threads();
  }
  return t;
#else
  return 1;
#endif
}

unsigned long long orc_ring_perm_closed(unsigned long long i, int n, int inverse) {
  return ring_perm_closed(i, n, inverse != 0);
}

unsigned long long orc_ring_perm_loop(unsigned long long i, int n, int inverse) {
  return ring_perm_loop(i, n, inverse != 0);
}

// Final state (interleaved re,im; 2*2^n doubles).  gate_level selects the
// PennyLane gate-by-gate circuit instead of the structured schedule.
int orc_forward_state(int n, int L, const double *params, int gate_level, double *out) {
  if (!valid_shape(n, L) || params == nullptr || out == nullptr) return 1;
  set_threads();
  const std::size_t S = std::size_t{1} << n;
  std::vector<cplx> cur(S);
  if (gate_level) {
    gate_level_forward(cur, n, L, params);
  } else {
    std::vector<cplx> scratch(S);
    structured_forward(cur, scratch, n, L, params);
  }
  std::memcpy(out, cur.data(), S * sizeof(cplx));
  return 0;
}

// lambda = H psi for an arbitrary state; returns <psi|H|psi> in *energy.
int orc_apply_hamiltonian(int n, double field, const double *state, double *out,
                          double *energy) {
  if (n < 2 || n > 34 || state == nullptr || out == nullptr) return 1;
  set_threads();
  const double e = apply_hamiltonian_energy(reinterpret_cast<cplx *>(out),
                                            reinterpret_cast<const cplx *>(state), n, field);
  if (energy != nullptr) *energy = e;
  return 0;
}

// Energy and gradient.  mode 0 = structured_adjoint (the reference's
// schedule), mode 1 = gate-level inverse walk (RZ^-1 then RY^-1 per wire).
// gradient may be null (energy only).
int orc_energy_and_grad(int n, int L, double field, const double *params, int mode,
                        double *energy, double *gradient) {
  if (!valid_shape(n, L) || params == nullptr || energy == nullptr) return 1;
  set_threads();
  const std::size_t S = std::size_t{1} << n;
  std::vector<cplx> cur(S), lam(S), scratch(S);
  if (mode == 0) {
    structured_forward(cur, scratch, n, L, params);
  } else {
    gate_level_forward(cur, n, L, params);
  }
  *energy = apply_hamiltonian_energy(lam.data(), cur.data(), n, field);
  if (gradient == nullptr) return 0;
  const std::size_t np = static_cast<std::size_t>(2) * n * L;
  std::fill(gradient, gradient + np, 0.0);
  if (mode == 0) {
    // cpp/ising_cuda_structured_adjoint_modes.inc:272-307: per layer, inverse
    // ring layer on psi and lambda, then wires high -> low.
    for (int layer = L; layer-- > 0;) {
      ring_gather_inverse(scratch.data(), cur.data(), n);
      std::swap(cur, scratch);
      ring_gather_inverse(scratch.data(), lam.data(), n);
      std::swap(lam, scratch);
      for (int w = n; w-- > 0;) {
        const std::size_t base = 2 * (static_cast<std::size_t>(layer) * n + w);
        ryrz_backward_wire(cur.data(), lam.data(), n, w,
                           make_coeffs(params[base], params[base + 1]), &gradient[base],
                           &gradient[base + 1]);
      }
    }
  } else {
    // cpp/ising_cuda_gate_level_adjoint_modes.inc:147-185: reverse gate walk.
    for (int layer = L; layer-- > 0;) {
      for (int w = n; w-- > 0;) {
        apply_cnot(cur.data(), n, w, (w + 1) % n);
        apply_cnot(lam.data(), n, w, (w + 1) % n);
      }
      for (int w = n; w-- > 0;) {
        const std::size_t base = 2 * (static_cast<std::size_t>(layer) * n + w);
        gradient[base + 1] += rz_gradient(cur.data(), lam.data(), n, w, params[base + 1]);
        apply_rz(cur.data(), n, w, params[base + 1], true);
        apply_rz(lam.data(), n, w, params[base + 1], true);
        gradient[base] += ry_gradient(cur.data(), lam.data(), n, w, params[base]);
        apply_ry(cur.data(), n, w, params[base], true);
        apply_ry(lam.data(), n, w, params[base], true);
      }
    }
  }
  return 0;
}

}  // extern "C"
