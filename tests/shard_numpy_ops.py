"""Numpy restatement of the sharded engine's per-rank operations (test
infrastructure: include/rsv_shard.h states each operation; this module
restates it from the global index map, without the closed forms the CUDA
kernels use).

It runs ``ShardedEngine`` on CPU tensors (multi-process ``gloo`` tests and
virtual ranks without a GPU), and each operation is the checker of its CUDA
kernel on the same inputs.  Conventions of the reference: bit w of the
amplitude index is wire w; per wire U = RZ(phi) RY(theta); one layer = U on
every wire, then CNOT(0,1), ..., CNOT(n-1,0) (cpp/ising_cuda_kernels.cu:22-25,
178-205); H = -sum Z_w Z_{w+1} - h sum X_w (cpp/ising_cuda_kernels.cu:313-358);
the gradient sums of the inverse walk (cpp/ising_cuda_gate_level_adjoint_
modes.inc:147-260).
"""

from __future__ import annotations

import numpy as np


def ring_map(x: np.ndarray, n: int) -> np.ndarray:
    """P(x) by the CNOT sequence CNOT(0,1), ..., CNOT(n-2,n-1), CNOT(n-1,0)."""
    x = np.asarray(x, dtype=np.uint64).copy()
    one = np.uint64(1)
    for w in range(n):
        c, t = np.uint64(w), np.uint64((w + 1) % n)
        x ^= ((x >> c) & one) << t
    return x


def ring_map_inv(y: np.ndarray, n: int) -> np.ndarray:
    """P^-1(y): the CNOT sequence in reverse."""
    y = np.asarray(y, dtype=np.uint64).copy()
    one = np.uint64(1)
    for w in range(n - 1, -1, -1):
        c, t = np.uint64(w), np.uint64((w + 1) % n)
        y ^= ((y >> c) & one) << t
    return y


def _bits(n: int) -> np.ndarray:
    return np.arange(1 << n, dtype=np.uint64)


class Geometry:
    """Global index <-> (rank, local offset) in layouts C and S."""

    def __init__(self, n: int, g: int) -> None:
        self.n, self.g = n, g
        self.nloc = n - g
        self.B = 1 << (n - 2 * g)
        self.N = 1 << g

    def global_c(self, rank: int) -> np.ndarray:
        return (np.uint64(rank) << np.uint64(self.nloc)) | _bits(self.nloc)

    def global_s(self, rank: int) -> np.ndarray:
        off = _bits(self.nloc)
        low = off & np.uint64(self.B - 1)
        top = off >> np.uint64(self.n - 2 * self.g)
        return low | (np.uint64(rank) << np.uint64(self.n - 2 * self.g)) | (top << np.uint64(self.nloc))

    def rank_c(self, x):
        return (x >> np.uint64(self.nloc)).astype(np.int64)

    def local_c(self, x):
        return (x & np.uint64((1 << self.nloc) - 1)).astype(np.int64)

    def rank_s(self, x):
        return ((x >> np.uint64(self.n - 2 * self.g)) & np.uint64(self.N - 1)).astype(np.int64)

    def local_s(self, x):
        low = x & np.uint64(self.B - 1)
        top = x >> np.uint64(self.nloc)
        return (low | (top << np.uint64(self.n - 2 * self.g))).astype(np.int64)


def _rot(a: np.ndarray, bit: int, c) -> None:
    """The forward gate on local bit `bit` of the vector a, in place, as the
    shard kernels apply it: (1/f) diag(1, e^{i phi}) RY(theta), f the larger in
    magnitude of cos(theta/2), sin(theta/2)."""
    ct, st, cp, sp = c
    f = ct if abs(ct) >= abs(st) else st
    v = a.reshape(-1, 2, 1 << bit)
    x0, x1 = v[:, 0, :].copy(), v[:, 1, :].copy()
    y0, y1 = (ct * x0 - st * x1) / f, (st * x0 + ct * x1) / f
    v[:, 0, :] = y0
    v[:, 1, :] = y1 * (cp + 1j * sp) ** 2


def _unrot(a: np.ndarray, l: np.ndarray, bit: int, c) -> tuple[float, float]:
    """Inverse walk of one wire on psi a and lambda l: (theta sum, phi sum)."""
    ct, st, cp, sp = c
    va, vl = a.reshape(-1, 2, 1 << bit), l.reshape(-1, 2, 1 << bit)
    a0, a1 = va[:, 0, :].copy(), va[:, 1, :].copy()
    l0, l1 = vl[:, 0, :].copy(), vl[:, 1, :].copy()
    gp = float(np.sum(np.imag(np.conj(l0) * a0)) - np.sum(np.imag(np.conj(l1) * a1)))
    ph = (cp - 1j * sp) ** 2  # diag(1, e^{-i phi}): RZ^dagger up to a common phase
    a1, l1 = a1 * ph, l1 * ph
    gt = float(np.sum(np.real(np.conj(l1) * a0)) - np.sum(np.real(np.conj(l0) * a1)))
    va[:, 0, :], va[:, 1, :] = ct * a0 + st * a1, ct * a1 - st * a0
    vl[:, 0, :], vl[:, 1, :] = ct * l0 + st * l1, ct * l1 - st * l0
    return gt, gp


class NumpyShardOps:
    """Same calls as ``CudaShardOps``, on CPU tensors."""

    def check(self, n: int, g: int) -> None:
        if not (0 <= g <= 3 and n - 2 * g >= 12 and n - g <= 31):
            raise ValueError("unsupported sharded geometry")

    def scratch_doubles(self, n: int, g: int) -> int:
        return 1

    @staticmethod
    def _coef(coef, layer, n, w):
        c = coef.numpy().reshape(-1, 4)[layer * n + w]
        return float(c[0]), float(c[1]), float(c[2]), float(c[3])

    def coef(self, n, L, params, coef):
        p = params.numpy().reshape(-1, 2)
        c = coef.numpy().reshape(-1, 4)
        c[:, 0], c[:, 1] = np.cos(p[:, 0] / 2), np.sin(p[:, 0] / 2)
        c[:, 2], c[:, 3] = np.cos(p[:, 1] / 2), np.sin(p[:, 1] / 2)

    def init(self, n, g, rank, psi):
        a = psi.numpy()
        a[:] = 0
        if rank == 0:
            a[0] = 1.0

    def rotate_local(self, n, g, layer, coef, psi):
        a = psi.numpy()
        for w in range(n - g):
            _rot(a, w, self._coef(coef, layer, n, w))

    def rotate_local_adjoint(self, n, g, L, layer, coef, psi, lam, scratch, result):
        a, l, r = psi.numpy(), lam.numpy(), result.numpy()
        for w in range(n - g):
            gt, gp = _unrot(a, l, w, self._coef(coef, layer, n, w))
            r[2 + 2 * (layer * n + w)] = gt
            r[2 + 2 * (layer * n + w) + 1] = gp

    def energy_local(self, n, g, rank, field, psi, lam, scratch, result):
        G = Geometry(n, g)
        y = G.global_c(rank)
        a, lm = psi.numpy(), lam.numpy()
        diag = np.zeros(y.shape, dtype=np.float64)
        for w in range(n):
            zw = 1 - 2 * ((y >> np.uint64(w)) & np.uint64(1)).astype(np.int64)
            zn = 1 - 2 * ((y >> np.uint64((w + 1) % n)) & np.uint64(1)).astype(np.int64)
            diag -= zw * zn
        out = diag * a
        idx = np.arange(a.size)
        for w in range(n - g):
            out = out - field * a[idx ^ (1 << w)]
        lm[:] = out
        result.numpy()[0] = float(np.real(np.vdot(a, out)))

    def ring_pack(self, n, g, rank, layer, coef, psi_s, send):
        G = Geometry(n, g)
        a = psi_s.numpy().copy()
        cf = coef.numpy().reshape(-1, 4)[layer * n:(layer + 1) * n]
        a *= float(np.prod(np.where(np.abs(cf[:, 0]) >= np.abs(cf[:, 1]), cf[:, 0], cf[:, 1])))
        for j in range(g):
            _rot(a, n - 2 * g + j, self._coef(coef, layer, n, n - g + j))
        x = G.global_s(rank)
        y = ring_map(x, n)
        dest = G.rank_c(y) * G.B + (x & np.uint64(G.B - 1)).astype(np.int64)
        out = send.numpy()
        out[dest] = a

    def ring_unpack(self, n, g, rank, recv, psi_c):
        G = Geometry(n, g)
        y = G.global_c(rank)
        x = ring_map_inv(y, n)
        src = G.rank_s(x) * G.B + (x & np.uint64(G.B - 1)).astype(np.int64)
        psi_c.numpy()[:] = recv.numpy()[src]

    def ring_pack_adjoint(self, n, g, rank, psi_c, lam_c, send_psi, send_lam):
        G = Geometry(n, g)
        y = G.global_c(rank)
        x = ring_map_inv(y, n)
        dest = G.rank_s(x) * G.B + (x & np.uint64(G.B - 1)).astype(np.int64)
        send_psi.numpy()[dest] = psi_c.numpy()
        send_lam.numpy()[dest] = lam_c.numpy()

    def ring_unpack_adjoint(self, n, g, rank, L, layer, coef, field, add_field, recv_psi, recv_lam, psi_s, lam_s,
                            scratch, result):
        G = Geometry(n, g)
        x = G.global_s(rank)
        y = ring_map(x, n)
        src = G.rank_c(y) * G.B + (x & np.uint64(G.B - 1)).astype(np.int64)
        a = recv_psi.numpy()[src].copy()
        lm = recv_lam.numpy()[src].copy()
        if add_field:
            add = np.zeros_like(a)
            for w in range(n - g, n):
                e = np.uint64(1) << np.uint64(w)
                mask = ring_map_inv(np.array([e], dtype=np.uint64), n)[0]
                partner = x ^ mask
                assert np.all(G.rank_s(partner) == rank)
                add += a[G.local_s(partner)]
            lm -= field * add
            result.numpy()[1] = float(np.real(np.vdot(a, -field * add)))
        if layer >= 0:
            r = result.numpy()
            for j in range(g):
                w = n - g + j
                gt, gp = _unrot(a, lm, n - 2 * g + j, self._coef(coef, layer, n, w))
                r[2 + 2 * (layer * n + w)] = gt
                r[2 + 2 * (layer * n + w) + 1] = gp
        psi_s.numpy()[:] = a
        lam_s.numpy()[:] = lm
