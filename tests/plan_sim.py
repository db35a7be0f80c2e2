"""Numpy execution of the engine's pass plan (host-logic check, no GPU).

``librsv.so`` describes the launch sequence it would run (``rsv_describe_plan``):
every pass's tile directions, gated wires, load/store modes (natural, gather
through P, scatter through P or P^-1, analytic product state), RZ-phase and
phi-gradient flags and buffer ids.  This module executes that description
with whole-state numpy operations, using the same algebra as the CUDA
kernels (RZ folded into one phase per amplitude per layer, theta gradient
Re(conj(lam1) psi0) - Re(conj(lam0) psi1) in the RZ-free frame, phi gradient
tot - 2*B_w), and also enumerates every tile/thread/register index of each
pass to check that a pass touches every amplitude exactly once.  Tests
compare the result with the oracle.
"""

from __future__ import annotations

import ctypes
import re

import numpy as np

from gpu_simulation_b200._lib import load_library


AUTO, UNCOMPUTE, CHECKPOINT = 0, 1, 2  # RSV_BACKWARD_* of include/rsv.h


def describe_plan(n: int, layers: int, mode: int = AUTO) -> str:
    lib = load_library()
    buf = ctypes.create_string_buffer(1 << 20)
    ln = ctypes.c_size_t()
    rc = lib.rsv_describe_plan_mode(n, layers, mode, buf, len(buf), ctypes.byref(ln))
    if rc != 0:
        raise ValueError(lib.rsv_last_error().decode())
    return buf.value.decode()


_STEP = re.compile(
    r"(?P<dir>fwd|bwd) layer=(?P<layer>\d+)(?: pass=(?P<pass>\d+))? dirs=\[(?P<dirs>[^\]]*)\] "
    r"gates=\[(?P<gates>[^\]]*)\] runs=\[(?P<runs>[^\]]*)\] tiles=(?P<tiles>\d+) "
    r"psi:(?P<pl>[\w()]+)\((?P<pi>-?\d+)\)->(?P<ps>\w+)\((?P<po>-?\d+)\)"
    r"(?: lam:(?P<ll>[\w()]+)\((?P<li>-?\d+)\)->(?P<ls>\w+)\((?P<lo>-?\d+)\))?"
    r"(?P<flags>.*) grid=(?P<grid>\d+)"
)


def parse_plan(text: str) -> dict:
    lines = text.strip().splitlines()
    head = dict(kv.split("=") for kv in lines[0].split())
    steps = []
    energy = None
    layer0 = None
    mps = None
    for ln in lines[1:]:
        if ln.startswith("mps "):
            m0 = re.match(r"mps K=(\d+) fwd psi:(\w+)\((-?\d+)\) grid=(\d+)", ln)
            if m0:
                steps.append(dict(kind="mps_fwd", K=int(m0[1]), store=m0[2], out=int(m0[3]), grid=int(m0[4])))
                continue
            m0 = re.match(r"mps K=(\d+) grad lam:(\w+)\((-?\d+)\) grid=(\d+)", ln)
            if not m0:
                raise ValueError(f"cannot parse plan line: {ln}")
            mps = dict(K=int(m0[1]), load=m0[2], buf=int(m0[3]), grid=int(m0[4]))
            continue
        if ln.startswith("layer0"):
            m0 = re.match(r"layer0 lam:(\w+)\((-?\d+)\) grid=(\d+)", ln)
            if not m0:
                raise ValueError(f"cannot parse plan line: {ln}")
            layer0 = dict(load=m0[1], buf=int(m0[2]), grid=int(m0[3]))
            continue
        if ln.startswith("energy"):
            kv = dict(x.split("=") for x in ln.split()[1:])
            energy = (int(kv["chi"]), int(kv["mu"]))
            continue
        if ln.startswith("finalize"):
            continue
        m = _STEP.match(ln)
        if not m:
            raise ValueError(f"cannot parse plan line: {ln}")
        dirs = []
        for d in m["dirs"].split(","):
            dirs.append(int(d, 16) if d.startswith("0x") else (1 << int(d)))
        gates = [int(g) for g in m["gates"].split(",") if g]
        runs = [tuple(int(x) for x in r.split(":")) for r in m["runs"].split(",") if r]
        steps.append(dict(
            bwd=m["dir"] == "bwd", layer=int(m["layer"]),
            pass_index=int(m["pass"]) if m["pass"] else -1,
            dirs=dirs, gates=gates, runs=runs, tiles=int(m["tiles"]),
            psi_load=m["pl"], psi_in=int(m["pi"]), psi_store=m["ps"], psi_out=int(m["po"]),
            lam_load=m["ll"], lam_in=int(m["li"]) if m["li"] else -1,
            lam_store=m["ls"], lam_out=int(m["lo"]) if m["lo"] else -1,
            phase=" phase" in m["flags"], phi=" phi" in m["flags"], grid=int(m["grid"]),
        ))
    return dict(n=int(head["n"]), L=int(head["L"]), phys=int(head["phys"]), steps=steps,
                energy=energy, bufs=int(head["bufs"]), mode=head["mode"], layer0=layer0,
                mps=mps)


def ring_p(i: np.ndarray, n: int) -> np.ndarray:
    mask = (1 << n) - 1
    lo = i & mask
    pre = lo.copy()
    for s in (1, 2, 4, 8, 16):
        pre ^= pre << s
    pre &= mask
    par = np.zeros_like(lo)
    x = lo >> 1
    while np.any(x):
        par ^= x & 1
        x >>= 1
    return (i & ~mask) | (pre & ~1) | par


def ring_pinv(j: np.ndarray, n: int) -> np.ndarray:
    mask = (1 << n) - 1
    lo = j & mask
    t = (lo ^ (lo << 1)) & mask
    t = np.where((lo >> (n - 1)) & 1, t ^ 3, t)
    return (j & ~mask) | t


def tile_indices(step: dict) -> np.ndarray:
    """Physical index of every (tile, thread, register) of a pass, computed
    the way the kernel does (deposit + XOR of tile directions)."""
    tiles = np.arange(step["tiles"], dtype=np.int64)
    base = np.zeros_like(tiles)
    rem = tiles.copy()
    for start, ln in step["runs"]:
        base |= (rem & ((1 << ln) - 1)) << start
        rem >>= ln
    t = np.arange(1 << len(step["dirs"]), dtype=np.int64)
    off = np.zeros_like(t)
    for b, v in enumerate(step["dirs"]):
        off ^= np.where((t >> b) & 1, v, 0)
    return (base[:, None] ^ off[None, :]).reshape(-1)


def check_pair_roles(step: dict, n: int) -> None:
    """The kernel rotates register pairs along tile bit b as (|0>, |1>) of the
    gated wire w, swapping the roles where the tile's multi-bit direction
    (flip bit) has coordinate 1.  Check that rule against the physical bit w
    of every element of every tile."""
    dirs = step["dirs"]
    flip = len(dirs)
    for b, v in enumerate(dirs):
        if v & (v - 1) and any((v >> w) & 1 for w in step["gates"]):
            flip = b
    ids = tile_indices(step).reshape(step["tiles"], 1 << len(dirs))
    t = np.arange(1 << len(dirs), dtype=np.int64)
    flip_coord = (t >> flip) & 1 if flip < len(dirs) else np.zeros_like(t)
    for w in step["gates"]:
        b = [i for i, v in enumerate(dirs) if v == (1 << w)]
        assert len(b) == 1, "a gated wire needs its unit direction in the tile"
        expected = ((t >> b[0]) & 1) ^ flip_coord
        actual = (ids >> w) & 1
        if not np.array_equal(actual, np.broadcast_to(expected, actual.shape)):
            raise AssertionError(f"pair roles of wire {w} disagree with the kernel rule: {step}")


def simulate(n: int, layers: int, field: float, params: np.ndarray, check_indices: bool = True,
             mode: int = AUTO):
    """Run the plan with numpy.  Returns (energy, gradient flat f64[2nL])."""
    plan = parse_plan(describe_plan(n, layers, mode))
    phys = plan["phys"]
    size = 1 << phys
    p = np.asarray(params, dtype=np.float64).reshape(layers, n, 2)
    c, s = np.cos(p[..., 0] * 0.5), np.sin(p[..., 0] * 0.5)
    ch, sh = np.cos(p[..., 1] * 0.5), np.sin(p[..., 1] * 0.5)
    idx = np.arange(size, dtype=np.int64)
    bits = (idx[:, None] >> np.arange(phys)[None, :]) & 1

    def phase(layer):
        ph = np.ones(size, dtype=np.complex128)
        for w in range(n):
            ph *= np.where(bits[:, w] == 1, ch[layer, w] + 1j * sh[layer, w], ch[layer, w] - 1j * sh[layer, w])
        return ph

    def product(j):
        amp = np.ones(j.shape, dtype=np.complex128)
        for w in range(phys):
            b = (j >> w) & 1
            if w < n:
                f0 = c[0, w] * (ch[0, w] - 1j * sh[0, w])
                f1 = s[0, w] * (ch[0, w] + 1j * sh[0, w])
                amp *= np.where(b == 1, f1, f0)
            else:
                amp *= np.where(b == 1, 0.0, 1.0)
        return amp

    def partial(j, mask):
        # layer-0 product state with only the wires in `mask` rotated (RY, no RZ)
        amp = np.ones(j.shape, dtype=np.complex128)
        for w in range(n):
            b = (j >> w) & 1
            if (mask >> w) & 1:
                amp *= np.where(b == 1, s[0, w], c[0, w])
            else:
                amp *= np.where(b == 1, 0.0, 1.0)
        return amp

    bufs = [np.zeros(size, dtype=np.complex128) for _ in range(plan["bufs"])]

    def load(mode, bid):
        if mode.startswith("partial("):
            return partial(idx, int(mode[len("partial("):-1], 16))
        if mode == "load":
            return bufs[bid].copy()
        if mode == "gatherP":
            return bufs[bid][ring_p(idx, n)]
        if mode == "product(P)":
            return product(ring_pinv(idx, n))
        if mode == "product":
            return product(idx)
        if mode == "mpsP":
            # the first K layers (their last ring applied), evaluated by the pass itself
            K = plan["mps"]["K"]
            chi = chi_k([[ry_rz(p[k, w, 0], p[k, w, 1]) for w in range(n)] for k in range(K)])
            return chi[ring_pinv(idx, n)]
        raise ValueError(mode)

    def store(mode, bid, v):
        if mode == "store":
            bufs[bid][:] = v
        elif mode == "scatterP":
            out = np.empty_like(v)
            out[ring_p(idx, n)] = v
            bufs[bid][:] = out
        elif mode == "scatterPinv":
            out = np.empty_like(v)
            out[ring_pinv(idx, n)] = v
            bufs[bid][:] = out
        elif mode != "none":
            raise ValueError(mode)

    theta = np.zeros((layers, n))
    phi = np.zeros((layers, n))
    energy = None

    def ry_rz(th, ph, dth=False, dph=False):
        cc, ss = np.cos(th / 2), np.sin(th / 2)
        ry = np.array([[-ss / 2, -cc / 2], [cc / 2, -ss / 2]]) if dth else np.array([[cc, -ss], [ss, cc]])
        rz = np.diag([np.exp(-0.5j * ph), np.exp(0.5j * ph)])
        if dph:
            rz = rz @ np.diag([-0.5j, 0.5j])
        return rz @ ry

    def chi_k(gates):
        # gates[k][w]: the 2x2 gate of layer k on wire w; output of the last
        # given layer before its CNOT ring
        amp0 = np.ones(size, dtype=np.complex128)
        for w in range(phys):
            b = bits[:, w]
            if w < n:
                amp0 *= np.where(b == 1, gates[0][w][1, 0], gates[0][w][0, 0])
            else:
                amp0 *= np.where(b == 1, 0.0, 1.0)
        out = amp0
        for k in range(1, len(gates)):
            nxt = np.zeros(size, dtype=np.complex128)
            nxt[ring_p(idx, n)] = out
            out = nxt
            for w in range(n):
                m = 1 << w
                lo = idx[(idx & m) == 0]
                x0, x1 = out[lo].copy(), out[lo | m].copy()
                u = gates[k][w]
                out[lo], out[lo | m] = u[0, 0] * x0 + u[0, 1] * x1, u[1, 0] * x0 + u[1, 1] * x1
        return out

    def energy_step():
        chi_b, mu_b = plan["energy"]
        chi = bufs[chi_b]
        real = idx < (1 << n)
        pi = ring_p(idx, n) & ((1 << n) - 1)
        rot = ((pi << 1) & ((1 << n) - 1)) | (pi >> (n - 1))
        walls = np.zeros(size, dtype=np.int64)
        x = pi ^ rot
        for w in range(n):
            walls += (x >> w) & 1
        mu = (2.0 * walls - n) * chi
        for w in range(n):
            mu = mu - field * chi[idx ^ int(ring_pinv(np.array([1 << w]), n)[0])]
        mu = np.where(real, mu, 0.0)
        bufs[mu_b][:] = mu
        return float(np.sum((np.conj(chi) * mu).real))

    for st in plan["steps"]:
        if st.get("kind") == "mps_fwd":
            # the first K layers, before the last one's ring, by direct simulation
            store(st["store"], st["out"], chi_k([[ry_rz(p[k, w, 0], p[k, w, 1]) for w in range(n)]
                                                 for k in range(st["K"])]))
            continue
        if check_indices:
            ids = tile_indices(st)
            if ids.size != size or not np.array_equal(np.sort(ids), idx):
                raise AssertionError(f"pass does not cover the state exactly once: {st}")
            check_pair_roles(st, n)
        layer = st["layer"]
        if not st["bwd"]:
            a = load(st["psi_load"], st["psi_in"])
            for w in st["gates"]:
                m = 1 << w
                lo = idx[(idx & m) == 0]
                a0, a1 = a[lo].copy(), a[lo | m].copy()
                a[lo] = c[layer, w] * a0 - s[layer, w] * a1
                a[lo | m] = s[layer, w] * a0 + c[layer, w] * a1
            if st["phase"]:
                a = a * phase(layer)
            store(st["psi_store"], st["psi_out"], a)
            continue
        if energy is None:
            energy = energy_step()
        a = load(st["psi_load"], st["psi_in"])
        b = load(st["lam_load"], st["lam_in"])
        if st["phase"]:
            ph = np.conj(phase(layer))
            a, b = a * ph, b * ph
        if st["phi"]:
            q = (np.conj(b) * a).imag
            tot = q.sum()
            for w in range(n):
                phi[layer, w] = tot - 2.0 * q[bits[:, w] == 1].sum()
        for w in st["gates"]:
            m = 1 << w
            lo = idx[(idx & m) == 0]
            a0, a1, b0, b1 = a[lo].copy(), a[lo | m].copy(), b[lo].copy(), b[lo | m].copy()
            theta[layer, w] = np.sum((np.conj(b1) * a0).real - (np.conj(b0) * a1).real)
            cc, ss = c[layer, w], s[layer, w]
            a[lo], a[lo | m] = cc * a0 + ss * a1, -ss * a0 + cc * a1
            b[lo], b[lo | m] = cc * b0 + ss * b1, -ss * b0 + cc * b1
        store(st["psi_store"], st["psi_out"], a)
        store(st["lam_store"], st["lam_out"], b)
    if energy is None:
        energy = energy_step()
    if plan["layer0"] is not None:
        # layer 0 from lambda alone: 2 Re <lambda0 | d psi0>, psi0 the product state
        l0 = plan["layer0"]
        lam0 = load(l0["load"], l0["buf"])
        a0 = c[0] * (ch[0] - 1j * sh[0])  # a_w(0)
        a1 = s[0] * (ch[0] + 1j * sh[0])  # a_w(1)
        for w in range(n):
            rest = np.ones(size, dtype=np.complex128)
            for v in range(n):
                if v != w:
                    rest *= np.where(bits[:, v] == 1, a1[v], a0[v])
            rest = np.where(idx < (1 << n), rest, 0.0)
            cl = np.conj(lam0) * rest
            S0, S1 = cl[bits[:, w] == 0].sum(), cl[bits[:, w] == 1].sum()
            e_m, e_p = ch[0, w] - 1j * sh[0, w], ch[0, w] + 1j * sh[0, w]
            dt0, dt1 = -0.5 * s[0, w] * e_m, 0.5 * c[0, w] * e_p
            dp0, dp1 = -0.5j * a0[w], 0.5j * a1[w]
            theta[0, w] = 2.0 * (dt0 * S0 + dt1 * S1).real
            phi[0, w] = 2.0 * (dp0 * S0 + dp1 * S1).real
    if plan["mps"] is not None:
        # the first K layers from lambda at their output: 2 Re <lambda | d chi_K>
        mp = plan["mps"]
        K = mp["K"]
        lamk = load(mp["load"], mp["buf"])
        base = [[ry_rz(p[k, w, 0], p[k, w, 1]) for w in range(n)] for k in range(K)]
        for k in range(K):
            for w in range(n):
                for dth, dph in ((True, False), (False, True)):
                    g = [list(row) for row in base]
                    g[k][w] = ry_rz(p[k, w, 0], p[k, w, 1], dth, dph)
                    val = 2.0 * np.sum(np.conj(lamk) * chi_k(g)).real
                    (theta if dth else phi)[k, w] = val
    grad = np.stack([theta, phi], axis=-1).reshape(-1)
    return energy, grad
