"""numpy emulator of the fused pass kernel (logosq_b200/csrc/fused.cu), driven by
the program that lq_plan_dump returns.  It mirrors the kernel step by step --
tile gather in the TMA 128-byte-swizzled layout, per-round thread/element
addressing, register ops with their control/fix/pattern rules -- so the
planner and encoder can be checked against the oracle on the CPU."""
from __future__ import annotations

import ctypes as C

import numpy as np

from logosq_b200 import abi
from logosq_b200._lib import call

ROUND_DT = np.dtype([("eoff", np.int32, 16), ("gpos", np.uint64, 4), ("lane", np.int32, 12),
                     ("nlane", np.int32), ("op_begin", np.int32), ("op_end", np.int32),
                     ("pad", np.int32)], align=True)
OP_DT = np.dtype([("type", np.int32), ("k0", np.int32), ("k1", np.int32), ("cm", np.int32),
                  ("gmask", np.uint64), ("fixmask", np.uint64), ("pb0", np.int32),
                  ("pb1", np.int32), ("npat", np.int32), ("coef", np.int32),
                  ("param", np.int32), ("coef_alt", np.int32), ("param2", np.int32),
                  ("coef_alt2", np.int32)], align=True)

(F_M1, F_M1C, F_X, F_XC, F_DIAG, F_SWAP, F_M2, F_BLOCK3, F_BLOCK4, F_M2R, F_DTAB, F_R1S,
 F_PAIR) = range(13)


def dump(n, gates, theta=None):
    th = None if theta is None else np.ascontiguousarray(theta, dtype=np.float64)
    used = C.c_size_t()
    args = (n, abi.gate_ptr(gates), len(gates), None if th is None else abi.f64_ptr(th),
            0 if th is None else len(th))
    from logosq_b200._lib import lib
    lib().lq_plan_dump(*args, None, 0, C.byref(used))
    buf = np.zeros(used.value, dtype=np.uint8)
    call("lq_plan_dump", *args, buf.ctypes.data_as(C.c_void_p), used.value, C.byref(used))
    off = 0
    counts = np.frombuffer(buf, np.int32, 5, off)
    off += 20
    nst, nrd, nop, ncf, T = (int(x) for x in counts)
    steps = np.frombuffer(buf, np.int32, 5 * nst, off).reshape(nst, 5)
    off += 20 * nst
    rounds = np.frombuffer(buf, ROUND_DT, nrd, off)
    off += ROUND_DT.itemsize * nrd
    ops = np.frombuffer(buf, OP_DT, nop, off)
    off += OP_DT.itemsize * nop
    coef = np.frombuffer(buf, np.float64, ncf, off)
    return T, steps, rounds, ops, coef


def swz(i):
    return i ^ ((i >> 3) & 7)


def run(n, gates, psi, theta=None):
    """Apply the planned program to psi (complex128) exactly as the kernel would;
    standalone steps use the oracle for that single gate."""
    import oracle
    T, steps, rounds, ops, coef = dump(n, gates, theta)
    m = T - 4
    psi = psi.copy()
    nthreads = 1 << (T - 4)
    tid = np.arange(nthreads)
    for st in steps:
        fused, gate, h = int(st[0]), int(st[1]), int(st[2])
        if not fused:
            oracle.apply_circuit(psi, gates[gate:gate + 1], theta)
            continue
        rb, nr = int(st[3]), int(st[4])
        # global index of local tile index l: low 4 bits, then bits h..h+m-1
        loc = np.arange(1 << T)
        g_of_l = (loc & 15) | ((loc >> 4) << h)
        ntiles = 1 << (n - T)
        for bid in range(ntiles):
            c2 = bid & ((1 << (h - 4)) - 1)
            c4 = bid >> (h - 4)
            tile_base = (c2 << 4) | (c4 << (h + m))
            gidx = tile_base | g_of_l
            smem = np.empty(1 << T, dtype=np.complex128)
            smem[swz(loc)] = psi[gidx]  # TMA with 128-byte swizzle
            for r in range(rb, rb + nr):
                rd = rounds[r]
                tbase = np.zeros(nthreads, dtype=np.int64)
                for j in range(int(rd["nlane"])):
                    tbase |= ((tid >> j) & 1) << int(rd["lane"][j])
                sb = swz(tbase) << 4
                gbase = tile_base | (tbase & 15) | ((tbase >> 4) << h)
                slots = [((sb ^ int(rd["eoff"][e])) >> 4) for e in range(16)]
                a = [smem[s].copy() for s in slots]
                gp = [int(x) for x in rd["gpos"]]
                for o in range(int(rd["op_begin"]), int(rd["op_end"])):
                    apply_op(a, ops[o], coef, gbase, gp)
                for e in range(16):
                    smem[slots[e]] = a[e]
            psi[gidx] = smem[swz(loc)]
    return psi


def apply_op(a, op, coef, gbase, gp):
    t = int(op["type"])
    gmask = int(op["gmask"])
    act = (gbase & gmask) == gmask
    c = coef[int(op["coef"]):]

    def cpx(k):
        return complex(c[2 * k], c[2 * k + 1])

    k0, k1, cm = int(op["k0"]), int(op["k1"]), int(op["cm"])
    if t in (F_M1, F_M1C, F_X, F_XC):
        K = k0
        for e in range(16):
            if e & (1 << K):
                continue
            if t in (F_M1C, F_XC) and (e & cm) != cm:
                continue
            a0, a1 = a[e], a[e | (1 << K)]
            if t in (F_M1, F_M1C):
                n0 = cpx(0) * a0 + cpx(1) * a1
                n1 = cpx(2) * a0 + cpx(3) * a1
            else:
                n0, n1 = a1, a0
            a[e] = np.where(act, n0, a0)
            a[e | (1 << K)] = np.where(act, n1, a1)
    elif t == F_DIAG:
        fm = int(op["fixmask"])
        pb0, pb1, npat = int(op["pb0"]), int(op["pb1"]), int(op["npat"])
        ph = np.array([cpx(k) for k in range(4)])
        for e in range(16):
            gi = gbase.copy()
            for k in range(4):
                if e >> k & 1:
                    gi |= gp[k]
            cond = ((gi & fm) == fm) & act
            b0 = (gi >> pb0) & 1 if npat > 0 else 0
            b1 = (gi >> pb1) & 1 if npat > 1 else 0
            a[e] = np.where(cond, a[e] * ph[b0 + 2 * b1], a[e])
    elif t == F_SWAP:
        for e in range(16):
            if (e & (1 << k0)) and not (e & (1 << k1)):
                f = e ^ (1 << k0) ^ (1 << k1)
                x, y = a[e], a[f]
                a[e] = np.where(act, y, x)
                a[f] = np.where(act, x, y)
    elif t == F_M2:
        M = np.array([cpx(k) for k in range(16)]).reshape(4, 4)
        for e in range(16):
            if (e & (1 << k0)) or (e & (1 << k1)):
                continue
            idx = [e, e | (1 << k1), e | (1 << k0), e | (1 << k0) | (1 << k1)]
            vin = [a[i] for i in idx]
            for rr in range(4):
                out = sum(M[rr, q] * vin[q] for q in range(4))
                a[idx[rr]] = np.where(act, out, vin[rr])
    elif t == F_M2R:
        M = np.array([c[k] for k in range(16)]).reshape(4, 4)
        for e in range(16):
            if (e & (1 << k0)) or (e & (1 << k1)):
                continue
            idx = [e, e | (1 << k1), e | (1 << k0), e | (1 << k0) | (1 << k1)]
            vin = [a[i] for i in idx]
            for rr in range(4):
                out = sum(M[rr, q] * vin[q] for q in range(4))
                a[idx[rr]] = np.where(act, out, vin[rr])
    elif t == F_R1S:
        x = c[0]
        for e in range(16):
            if e & (1 << k0):
                continue
            a0, a1 = a[e], a[e | (1 << k0)]
            if k1 == 0:
                n0, n1 = a0 - x * a1, a1 + x * a0
            else:
                n0, n1 = x * a0 - a1, a0 + x * a1
            a[e] = np.where(act, n0, a0)
            a[e | (1 << k0)] = np.where(act, n1, a1)
    elif t == F_PAIR:
        def rot(y0, y1, x, form):
            if form == 0:
                return y0 - x * y1, y1 + x * y0
            return x * y0 - y1, y0 + x * y1
        f0, f1, perm = cm & 1, (cm >> 1) & 1, cm >> 2
        P = [[0, 1, 2, 3], [0, 1, 3, 2], [0, 3, 2, 1], [0, 2, 1, 3]][perm]
        for e in range(16):
            if (e & (1 << k0)) or (e & (1 << k1)):
                continue
            idx = [e, e | (1 << k1), e | (1 << k0), e | (1 << k0) | (1 << k1)]
            v = [a[i] for i in idx]
            v[0], v[1] = rot(v[0], v[1], c[1], f1)
            v[2], v[3] = rot(v[2], v[3], c[1], f1)
            v[0], v[2] = rot(v[0], v[2], c[0], f0)
            v[1], v[3] = rot(v[1], v[3], c[0], f0)
            old = [a[i] for i in idx]
            for q in range(4):
                a[idx[P[q]]] = np.where(act, v[q], old[P[q]])
    elif t == F_DTAB:
        npat, pb0, pb1 = int(op["npat"]), int(op["pb0"]), int(op["pb1"])
        v = np.zeros_like(gbase)
        if npat > 0:
            v = (gbase >> pb0) & 1
        if npat > 1:
            v = v | (((gbase >> pb1) & 1) << 1)
        tab = np.array([cpx(k) for k in range(16 << npat)]).reshape(1 << npat, 16)
        for e in range(16):
            a[e] = np.where(act, a[e] * tab[v, e], a[e])
    else:
        raise NotImplementedError(t)
