"""Executes the engine's lowered programs on the CPU (numpy, float64).

A checker for the host-side lowering: register allocation, trajectory saves and
the reverse schedule.  It supports the opcodes the lowering tests use and the
plain-value (gradient) kind.
"""
from __future__ import annotations

import ctypes
import math
import struct

import numpy as np

from echidna_b200 import _lib
from echidna_b200.tape import OpCode

INS = struct.Struct("<BBBBIIIIid")
RINS = struct.Struct("<BBHIIIIIIi")
TERM = struct.Struct("<BBHIIBBBBIIIIIId")   # PTerm, 48 bytes
GREC = struct.Struct("<IIHBBIdQ")            # GRec, 32 bytes
DOUT = struct.Struct("<IIBBHIIId")           # PDenseOut, 32 bytes
XI_LDIN, XI_STOUT, XI_MOV, XI_SEED, XI_STGRAD, XI_CHAIN = 64, 65, 66, 67, 68, 69
XI_NORM, XI_GATHER, XI_DENSE = 84, 85, 86
CK_X, CK_CX, CK_XC, CK_XY, CK_C = range(5)
CF = dict(X_INIT=1, Y_INIT=2, X_GLOB=4, Y_GLOB=8, X_ADJ=16, Y_ADJ=32)
M_SMEM, M_GLOB, M_IMM, M_NONE = 0, 1, 2, 3
NONE = 0xFFFFFFFF
RF = dict(R_GLOB=1, A_GLOB=2, B_GLOB=4, A_INIT=8, B_INIT=16, VA_IMM=32, VB_IMM=64, HAS_A=128, HAS_B=256)
KIND = {"forward": 0, "gradient": 1, "hvp": 2, "tangent": 3, "taylor": 4, "taylor_direct": 5}


def plan_dump(tape, kind: str, cap: int, dense_max: int = 16):
    lib = _lib.load()
    op, a0, a1, vals = tape.arrays()
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    outs = np.asarray(tape.output_indices, dtype=np.uint32)
    counts = (ctypes.c_uint64 * 9)()
    args = [_lib.ptr(op), _lib.ptr(a0), _lib.ptr(a1), _lib.ptr(vals), len(op), tape.num_inputs, tape.output_index,
            _lib.ptr(outs), len(outs), KIND[kind], cap]
    st = lib.ech_plan_dump(*args, None, 0, None, 0, None, 0, None, 0, None, 0, None, 0, dense_max, counts)
    assert st == 0, _lib.last_error()
    nf, nr, npool, nt, ng, nd = counts[0], counts[1], counts[2], counts[6], counts[7], counts[8]
    db = ctypes.create_string_buffer(max(nd, 1) * 32)
    gb = ctypes.create_string_buffer(max(ng, 1) * 32)
    fb = ctypes.create_string_buffer(max(nf, 1) * 32)
    rb = ctypes.create_string_buffer(max(nr, 1) * 32)
    tb = ctypes.create_string_buffer(max(nt, 1) * 48)
    pool = np.zeros(max(npool, 1), dtype=np.float64)
    st = lib.ech_plan_dump(*args, ctypes.addressof(fb), nf, ctypes.addressof(rb), nr, _lib.ptr(pool), npool,
                           ctypes.addressof(tb), nt, ctypes.addressof(gb), ng, ctypes.addressof(db), nd, dense_max,
                           counts)
    assert st == 0, _lib.last_error()
    fwd = [INS.unpack_from(fb, 32 * k) for k in range(nf)]
    rev = [RINS.unpack_from(rb, 32 * k) for k in range(nr)]
    terms = []
    for k in range(nt):
        (kind_, op_, flags, xs, ys, fxm, fym, rxm, rym, fxi, fyi, rxi, ryi, vx, vy, c) = TERM.unpack_from(tb, 48 * k)
        terms.append(dict(kind=kind_, op=op_, flags=flags, fxm=fxm, fym=fym, fxi=fxi, fyi=fyi, rxm=rxm, rym=rym,
                          rxi=rxi, ryi=ryi, vx=vx, vy=vy, c=c))
    gathers = []
    for k in range(ng):
        s, n, flags, mode, _pad, idx, c, _p2 = GREC.unpack_from(gb, 32 * k)
        gathers.append(dict(s=s, n=n, flags=flags, mode=mode, idx=idx, c=c))
    dense = []
    for k in range(nd):
        tb_, tn, am, dm, _pad, ai, di, save, a_val = DOUT.unpack_from(db, 32 * k)
        dense.append(dict(tb=tb_, tn=tn, am=am, dm=dm, ai=ai, di=di, save=save, a_val=a_val))
    return fwd, rev, pool, dict(smem_regs=counts[3], far_slots=counts[4], traj_slots=counts[5], terms=terms,
                                gathers=gathers, dense=dense)


def _fwd(op, a, b, aux):
    with np.errstate(all="ignore"):
        if op == OpCode.Add: return a + b
        if op == OpCode.Sub: return a - b
        if op == OpCode.Mul: return a * b
        if op == OpCode.Div: return a / b
        if op == OpCode.Neg: return -a
        if op == OpCode.Sin: return np.array([math.sin(v) for v in a])
        if op == OpCode.Cos: return np.array([math.cos(v) for v in a])
        if op == OpCode.Exp: return np.array([math.exp(v) for v in a])
        if op == OpCode.Tanh: return np.array([math.tanh(v) for v in a])
        if op == OpCode.Ln: return np.array([math.log(v) for v in a])
        if op == OpCode.Sqrt: return np.sqrt(a)
        if op == OpCode.Powi:
            out = np.empty_like(a)
            for i, v in enumerate(a):
                m, r, base = abs(aux), 1.0, v
                while True:
                    if m & 1:
                        r = r * base
                    m >>= 1
                    if m == 0:
                        break
                    base = base * base
                out[i] = 1.0 / r if aux < 0 else r
            return out
    raise NotImplementedError(OpCode(op).name)


def _partials(op, a, b, r, aux):
    one = np.ones_like(r if r is not None else a)
    zero = np.zeros_like(one)
    with np.errstate(all="ignore"):
        if op == OpCode.Add: return one, one
        if op == OpCode.Sub: return one, -one
        if op == OpCode.Mul: return b, a
        if op == OpCode.Div:
            inv = 1.0 / b
            return inv, -r * inv
        if op == OpCode.Neg: return -one, zero
        if op == OpCode.Sin: return np.array([math.cos(v) for v in a]), zero
        if op == OpCode.Cos: return -np.array([math.sin(v) for v in a]), zero
        if op == OpCode.Exp: return r, zero
        if op == OpCode.Tanh:
            c = np.array([math.cosh(v) for v in a])
            return 1.0 / (c * c), zero
        if op == OpCode.Ln: return np.where(a >= 0, 1.0 / a, np.nan), zero
        if op == OpCode.Sqrt: return 1.0 / ((1.0 + 1.0) * r), zero
        if op == OpCode.Powi:
            if aux == 0: return zero, zero
            return aux * _fwd(OpCode.Powi, a, None, aux - 1), zero
    raise NotImplementedError(OpCode(op).name)


def run_gradient(tape, X, cap, dense_max: int = 16):
    """Emulates the gradient programs; returns (outputs, grads)."""
    fwd, rev, pool, info = plan_dump(tape, "gradient", cap, dense_max)
    terms = info["terms"]
    X = np.asarray(X, dtype=np.float64)
    B = X.shape[0]
    regs = {M_SMEM: {}, M_GLOB: {}}
    traj = {}
    nout = len(tape.all_output_indices())
    outs = np.full((B, nout), np.nan)

    def ld(mode, idx, imm):
        if mode == M_IMM:
            return np.full(B, imm)
        return regs[mode][idx]

    for (opc, ma, mb, md, a, b, d, save, aux, imm) in fwd:
        if opc == XI_LDIN:
            v = X[:, aux].copy()
        elif opc == XI_STOUT:
            outs[:, aux] = ld(ma, a, imm)
            continue
        elif opc == XI_MOV:
            v = ld(ma, a, imm)
        elif opc == XI_DENSE:
            # every output's chain over the shared operands, results written
            # only after all operands are read (as the kernel does)
            results = []
            for o in info["dense"][a:a + aux]:
                acc = ld(o["am"], o["ai"], o["a_val"])
                for tm in terms[o["tb"]:o["tb"] + o["tn"]]:
                    x = regs[tm["fxm"]][tm["fxi"]]
                    with np.errstate(all="ignore"):
                        acc = acc + (tm["c"] * x if tm["kind"] == CK_CX else x * tm["c"])
                results.append((o, acc))
            for o, acc in results:
                regs[o["dm"]][o["di"]] = acc
                if o["save"] != NONE:
                    traj[o["save"]] = acc
            continue
        elif opc == XI_CHAIN:
            acc = ld(ma, a, imm)
            for tm in terms[b:b + aux]:
                k = tm["kind"]
                with np.errstate(all="ignore"):
                    if k == CK_C:
                        prod = np.full(B, tm["c"])
                    else:
                        x = regs[tm["fxm"]][tm["fxi"]]
                        if k == CK_X:
                            prod = x
                        elif k == CK_CX:
                            prod = tm["c"] * x
                        elif k == CK_XC:
                            prod = x * tm["c"]
                        else:
                            prod = x * regs[tm["fym"]][tm["fyi"]]
                    acc = [acc + prod, prod + acc, acc - prod, prod - acc][tm["op"]]
            v = acc
        else:
            av = ld(ma, a, imm)
            bv = np.zeros(B) if mb == M_NONE else ld(mb, b, imm)
            v = _fwd(opc, av, bv, aux)
        if md != M_NONE:
            regs[md][d] = v
        if save != NONE:
            traj[save] = v
    grads = np.full((B, tape.num_inputs), np.nan)
    regs = {M_SMEM: {}, M_GLOB: {}}
    for (opc, _pad, fl, r, a, b, va, vb, vr, aux) in rev:
        mr = M_GLOB if fl & RF["R_GLOB"] else M_SMEM
        if opc == XI_SEED:
            regs[mr][r] = np.ones(B)
            continue
        if opc == XI_STGRAD:
            grads[:, aux] = 0.0 if r == NONE else regs[mr][r]
            continue
        if opc == XI_GATHER:
            gathers = info["gathers"]
            q = va
            for _ in range(aux):
                hd = gathers[q]
                cur = np.zeros(B) if hd["flags"] & CF["X_INIT"] else regs[hd["mode"]][hd["idx"]]
                for g in gathers[q + 1:q + 1 + hd["n"]]:
                    t = regs[g["mode"]][g["idx"]]
                    hit = (t != 0) & (g["c"] != 0)
                    with np.errstate(all="ignore"):
                        cur = np.where(hit, cur + g["c"] * t, cur)
                regs[hd["mode"]][hd["idx"]] = cur
                q += 1 + hd["n"]
            continue
        adj = regs[mr][r]
        if opc == XI_NORM:
            with np.errstate(all="ignore"):
                regs[mr][r] = np.where(adj != 0, 0.0 + 1.0 * adj, 0.0)
            continue
        if opc == XI_CHAIN:
            adj_s = adj

            def acc_into(m, idx, init, d, a_):
                old = np.zeros(B) if init else regs[m][idx]
                hit = (a_ != 0) & (d != 0)
                with np.errstate(all="ignore"):
                    regs[m][idx] = np.where(hit, old + d * a_, old)

            for q in range(aux - 1, -1, -1):
                tm = terms[va + q]
                k = tm["kind"]
                sub = tm["op"] >= 2
                chain_a = (tm["op"] & 1) == 0
                one = np.ones(B)
                dA, dB = one, (-one if sub else one)
                d_acc, d_term = (dA, dB) if chain_a else (dB, dA)
                live = adj_s != 0
                new_prev = np.zeros(B)
                adj_p = np.zeros(B)

                def acc_side():
                    nonlocal new_prev
                    if q == 0 and fl & RF["HAS_A"]:
                        ma_ = M_GLOB if fl & RF["A_GLOB"] else M_SMEM
                        acc_into(ma_, a, fl & RF["A_INIT"], d_acc, adj_s)
                    else:
                        with np.errstate(all="ignore"):
                            new_prev = np.where(live & (d_acc != 0), 0.0 + d_acc * adj_s, 0.0)

                def term_side():
                    nonlocal adj_p
                    if k == CK_X:
                        mx = tm["rxm"]
                        acc_into(mx, tm["rxi"], tm["flags"] & CF["X_INIT"], d_term, adj_s)
                    elif k in (CK_CX, CK_XC, CK_XY):
                        with np.errstate(all="ignore"):
                            adj_p = np.where(live & (d_term != 0), 0.0 + d_term * adj_s, 0.0)

                if chain_a:
                    acc_side(); term_side()
                else:
                    term_side(); acc_side()
                if k in (CK_CX, CK_XC):
                    mx = tm["rxm"]
                    acc_into(mx, tm["rxi"], tm["flags"] & CF["X_INIT"], np.full(B, tm["c"]), adj_p)
                elif k == CK_XY:
                    xv = traj[tm["vx"]]
                    yv = traj[tm["vy"]]
                    mx = tm["rxm"]
                    my = tm["rym"]
                    acc_into(mx, tm["rxi"], tm["flags"] & CF["X_INIT"], yv, adj_p)
                    acc_into(my, tm["ryi"], tm["flags"] & CF["Y_INIT"], xv, adj_p)
                adj_s = new_prev
            continue

        def val(idx, is_imm):
            if idx == NONE:
                return np.zeros(B)
            return np.full(B, pool[idx]) if is_imm else traj[idx]

        A = val(va, fl & RF["VA_IMM"])
        Bv = val(vb, fl & RF["VB_IMM"])
        R = None if vr == NONE else traj[vr]
        da, db = _partials(opc, A, Bv, R if R is not None else np.zeros(B), aux)
        live = adj != 0
        for has, init, glob, idx, dd in ((RF["HAS_A"], RF["A_INIT"], RF["A_GLOB"], a, da),
                                         (RF["HAS_B"], RF["B_INIT"], RF["B_GLOB"], b, db)):
            if not fl & has:
                continue
            m = M_GLOB if fl & glob else M_SMEM
            old = np.zeros(B) if fl & init else regs[m][idx]
            hit = live & (dd != 0)
            with np.errstate(all="ignore"):
                new = np.where(hit, old + dd * adj, old)
            regs[m][idx] = new
    return outs, grads
