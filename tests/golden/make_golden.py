"""Generate tests/golden/golden_small.npz — small known-answer fixtures.

The reference (Fortran 2018 + HDF5 + spglib) cannot be compiled in this
environment and ships no golden vectors for the phonon-scattering path, so
these fixtures come from a second, independent restatement of the reference
written here in plain Python loops that transcribe the Fortran statement by
statement (slow; small sizes only).  The C++ oracle and the GPU library are
both checked against them.  Inputs that a different LAPACK build could change
(eigenvectors) are stored in the fixture next to the outputs.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


# --- TetrahedronQ_m.f90:56-221 / IndxChng_mod.f90:85-107 -------------------------
def py_make_tetrahedron(mesh, G, shift=(0, 0, 0)):
    box = [(0, 0, 0), (1, 0, 0), (0, 0, 1), (0, 1, 1), (1, 0, 1), (1, 1, 1), (1, 1, 0), (0, 1, 0)]
    nq = mesh[0] * mesh[1] * mesh[2]
    mesh_mul = (1, mesh[0], mesh[0] * mesh[1])
    Ru = [[G[r][i] / mesh[i] for i in range(3)] for r in range(3)]
    uniq = [True] * nq
    qint = [[0, 0, 0] for _ in range(nq)]
    qf = [[0.0, 0.0, 0.0] for _ in range(nq)]
    tets = []

    def fold(v):
        return [v[d] - mesh[d] if v[d] > mesh[d] // 2 else v[d] for d in range(3)]

    for iz in range(mesh[2]):
        for iy in range(mesh[1]):
            for ix in range(mesh[0]):
                vt = fold([ix, iy, iz])
                bt = []
                for v in range(8):
                    vert = [box[v][d] + vt[d] for d in range(3)]
                    vf = fold(vert)
                    g = sum((vf[d] % mesh[d]) * mesh_mul[d] for d in range(3)) + 1
                    bt.append(g)
                    if uniq[g - 1]:
                        qint[g - 1] = vf
                        qf[g - 1] = [sum(Ru[r][c] * (vf[c] + shift[c] * 0.5) for c in range(3)) for r in range(3)]
                        uniq[g - 1] = False
                pat = [(0, 1, 2, 3), (2, 3, 4, 1), (5, 3, 4, 1), (5, 3, 6, 1), (6, 3, 7, 1), (0, 3, 7, 1)]
                for p in pat:
                    tets.append([bt[k] for k in p])
    return np.array(qint, np.int32), np.array(qf), np.array(tets, np.int32)


def _gidx(v, mesh):
    return (v[0] % mesh[0]) + mesh[0] * (v[1] % mesh[1]) + mesh[0] * mesh[1] * (v[2] % mesh[2]) + 1


def _recp_latt(mesh):
    sgn = (0, 1, -1)
    out = []
    for c3 in range(3):
        for c2 in range(3):
            for c1 in range(3):
                out.append((sgn[c1] * mesh[0], sgn[c2] * mesh[1], sgn[c3] * mesh[2]))
    return out


def _within(bound, q, g, nq):
    return (not (any(q[d] > bound[d] for d in range(3)) or any(q[d] < -bound[d] for d in range(3)))) and 1 <= g <= nq


# --- QuasiMomentumConsrv3rd_m.f90:13-240 -------------------------------------------
def py_momentum3(mesh, qint, q0):
    nq = len(qint)
    bound = [m // 2 for m in mesh]
    covered = [False] * nq
    A = [[0, 0, 0, 0] for _ in range(nq)]
    perm = []
    cnt = tot = 0
    Gs = _recp_latt(mesh)
    for i1 in range(1, nq + 1):
        q1 = list(qint[i1 - 1])
        g1 = _gidx(q1, mesh)
        if covered[g1 - 1]:
            continue
        found = None
        for G in Gs:
            q2 = [G[d] - (q0[d] + q1[d]) for d in range(3)]
            g2 = _gidx(q2, mesh)
            if _within(bound, q2, g2, nq):
                found = (q2, g2)
                break
        if found is None:
            continue
        q2, g2 = found
        cnt += 1
        A[g1 - 1] = [1, cnt, g1, g2]
        covered[g1 - 1] = True
        tot += 1
        perm.append([g1, g2])
        # Permutation3rd: per = (2,1)
        if any((q2[d] - q1[d]) != 0 for d in range(3)) or any((q1[d] - q2[d]) != 0 for d in range(3)):
            A[g2 - 1] = [0, cnt, g2, g1]
            covered[g2 - 1] = True
            tot += 1
    return np.array(A, np.int32), np.array(perm, np.int32).reshape(-1, 2), (cnt, tot)


# --- QuasiMomentumConsrv4th_m.f90:32-312 -------------------------------------------
def py_momentum4(mesh, qint, q0):
    nq = len(qint)
    bound = [m // 2 for m in mesh]
    covered = np.zeros((nq, nq), bool)  # [q1][q2]
    A = np.zeros((nq, nq, 3), np.int32)
    perm = []
    cnt = tot = 0
    Gs = _recp_latt(mesh)
    per = [(1, 3, 2), (2, 1, 3), (2, 3, 1), (3, 1, 2), (3, 2, 1)]
    for i1 in range(1, nq + 1):
        q1 = list(qint[i1 - 1])
        g1 = _gidx(q1, mesh)
        for i2 in range(1, nq + 1):
            q2 = list(qint[i2 - 1])
            g2 = _gidx(q2, mesh)
            if covered[g1 - 1, g2 - 1]:
                continue
            found = None
            for G in Gs:
                q3 = [G[d] - (q0[d] + q1[d] + q2[d]) for d in range(3)]
                g3 = _gidx(q3, mesh)
                if _within(bound, q3, g3, nq):
                    found = (q3, g3)
                    break
            if found is None:
                continue
            q3, g3 = found
            cnt += 1
            A[g1 - 1, g2 - 1] = (0, cnt, g3)
            covered[g1 - 1, g2 - 1] = True
            tot += 1
            perm.append([g1, g2, g3])
            ini = [q1, q2, q3]
            gi = [g1, g2, g3]
            pg = []
            for pp in range(5):
                pq = [ini[per[pp][k] - 1] for k in range(3)]
                pgi = [gi[per[pp][k] - 1] for k in range(3)]
                pg.append(pgi)
                nonew = all(pq[k][d] - ini[k][d] == 0 for k in range(3) for d in range(3))
                for qq in range(pp):
                    nonew = nonew or all(pgi[k] - pg[qq][k] == 0 for k in range(3))
                if not nonew:
                    A[pgi[0] - 1, pgi[1] - 1] = (pp + 1, cnt, pgi[2])
                    covered[pgi[0] - 1, pgi[1] - 1] = True
                    tot += 1
    return A, np.array(perm, np.int32).reshape(-1, 3), (cnt, tot)


# --- TetrahedronIntegration_m.f90:18-218 (my_sort with its cyclic findloc search) ----
def py_my_sort(om, F, v1):
    omc, Fc, v1c = list(om), list(F), list(v1)
    srt = sorted(om)
    covered = [False] * 4
    F2, v2 = [0.0] * 4, [0] * 4
    for ii in range(4):
        strt = 0
        while True:
            strt = (strt + 1) % 4
            if strt == 0:
                strt = 4
            sub = omc[strt - 1:]
            idx = next((k + 1 for k, x in enumerate(sub) if x == srt[ii]), 0)
            act = strt + (idx - 1)
            if not covered[act - 1]:
                break
        covered[act - 1] = True
        v2[ii] = v1c[act - 1]
        F2[ii] = Fc[act - 1]
    return srt, F2, v2


def py_find_g_iver(Mqs, M, F, strict):
    M, F, perm = py_my_sort(M, F, [1, 2, 3, 4])
    if not strict:
        c1 = M[0] <= Mqs < M[1]
        c2 = M[1] <= Mqs < M[2]
        c3 = M[2] <= Mqs <= M[3]
    else:
        c1 = M[0] < Mqs < M[1]
        c2 = M[1] < Mqs < M[2]
        c3 = M[2] < Mqs < M[3]
    I = [0.0] * 4
    if c1:
        g = (3.0 * ((Mqs - M[0]) ** 2)) / ((M[1] - M[0]) * (M[2] - M[0]) * (M[3] - M[0]))
        I[0] = (((Mqs - M[1]) / (M[0] - M[1])) + ((Mqs - M[2]) / (M[0] - M[2])) + ((Mqs - M[3]) / (M[0] - M[3]))) / 3.0
        for v in range(1, 4):
            I[v] = ((Mqs - M[0]) / (M[v] - M[0])) / 3.0
        e = True
    elif c2:
        g = (3.0 / ((M[1] - M[2]) * (M[3] - M[0]))) * ((((Mqs - M[0]) * (Mqs - M[2])) / (M[2] - M[0]))
                                                       - (((Mqs - M[1]) * (Mqs - M[3])) / (M[1] - M[3])))
        den = g * (M[3] - M[0])
        I[0] = (((Mqs - M[3]) / (M[0] - M[3])) / 3.0) + ((((Mqs - M[2]) / (M[0] - M[2])) * ((Mqs - M[0]) / (M[2] - M[0]))
                                                            * ((Mqs - M[2]) / (M[1] - M[2]))) / den)
        I[1] = (((Mqs - M[2]) / (M[1] - M[2])) / 3.0) + (((((Mqs - M[3]) / (M[1] - M[3])) ** 2)
                                                            * ((Mqs - M[1]) / (M[2] - M[1]))) / den)
        I[2] = (((Mqs - M[1]) / (M[2] - M[1])) / 3.0) + (((((Mqs - M[0]) / (M[2] - M[0])) ** 2)
                                                            * ((Mqs - M[2]) / (M[1] - M[2]))) / den)
        I[3] = (((Mqs - M[0]) / (M[3] - M[0])) / 3.0) + ((((Mqs - M[1]) / (M[3] - M[1])) * ((Mqs - M[3]) / (M[1] - M[3]))
                                                            * ((Mqs - M[1]) / (M[2] - M[1]))) / den)
        e = True
    elif c3:
        g = (3.0 * ((Mqs - M[3]) ** 2)) / ((M[3] - M[0]) * (M[3] - M[1]) * (M[3] - M[2]))
        for v in range(3):
            I[v] = ((Mqs - M[3]) / (M[v] - M[3])) / 3.0
        I[3] = (((Mqs - M[0]) / (M[3] - M[0])) + ((Mqs - M[1]) / (M[3] - M[1])) + ((Mqs - M[2]) / (M[3] - M[2]))) / 3.0
        e = True
    else:
        g, e = 0.0, False
    return e, g, I, M, F, perm


# --- ThirdOrder_m.f90:278-439 (the 9-deep loop) --------------------------------------
def py_scatter_mat_el(q1, q2, q0chk, nb, fc3, num, btyp, posr, rsm, e0, e1, e2):
    """fc3[mu][N1][N2][a][b][c]; e*[s][row]; returns Phi[s][s1][s2] (complex)."""
    ndof = 3 * nb
    phi = [[[0j] * ndof for _ in range(ndof)] for _ in range(ndof)]
    strt = [4 if q0chk[i] else 1 for i in range(3)]
    for mu in range(nb):
        for N1 in range(int(num[mu])):
            nu = int(btyp[mu][N1]) - 1
            R1 = posr[mu][N1]
            qr1 = q1[0] * R1[0] + q1[1] * R1[1] + q1[2] * R1[2]
            ex1 = complex(math.cos(qr1), math.sin(qr1))
            for N2 in range(int(num[mu])):
                eta = int(btyp[mu][N2]) - 1
                R2 = posr[mu][N2]
                qr2 = q2[0] * R2[0] + q2[1] * R2[1] + q2[2] * R2[2]
                ex2 = complex(math.cos(qr2), math.sin(qr2))
                mf = rsm[mu] * rsm[nu] * rsm[eta]
                exm = ex1 * ex2 * mf
                for al in range(3):
                    r0 = 3 * mu + al
                    for s in range(strt[0] - 1, ndof):
                        w0 = e0[s][r0]
                        for be in range(3):
                            r1 = 3 * nu + be
                            for s1 in range(strt[1] - 1, ndof):
                                w1 = e1[s1][r1]
                                for ga in range(3):
                                    r2 = 3 * eta + ga
                                    pm = fc3[mu][N1][N2][al][be][ga] * exm
                                    for s2 in range(strt[2] - 1, ndof):
                                        phi[s][s1][s2] += pm * w0 * w1 * e2[s2][r2]
    return np.array(phi)


def main():
    from spring_b200 import synthetic as S
    from oracle import phonons as P
    from oracle import constants as C

    rng = np.random.default_rng(20241203)
    out = {}
    cr = S.build("rocksalt2")
    G = cr.G
    # mesh fixtures
    for N in (4, 5):
        qi, qf, tet = py_make_tetrahedron((N, N, N), G)
        out[f"mesh{N}_qint"], out[f"mesh{N}_qpnt"], out[f"mesh{N}_tet"] = qi, qf, tet
    # 3-phonon enumeration for every q0 of small meshes (even and odd)
    for N in (4, 5, 6):
        qi, _, _ = py_make_tetrahedron((N, N, N), G)
        As, Ps, Cs = [], [], []
        for q0 in qi:
            A, Pm, cnt = py_momentum3((N, N, N), qi, q0)
            As.append(A)
            Ps.append(np.pad(Pm, ((0, len(qi) - len(Pm)), (0, 0))))
            Cs.append(cnt)
        out[f"enum3_N{N}_A"] = np.array(As)
        out[f"enum3_N{N}_P"] = np.array(Ps)
        out[f"enum3_N{N}_C"] = np.array(Cs, np.int32)
    # 4-phonon enumeration, a few q0 on meshes 3 and 4
    for N in (3, 4):
        qi, _, _ = py_make_tetrahedron((N, N, N), G)
        sel = [0, 1, len(qi) // 2, len(qi) - 1]
        As, Ps, Cs = [], [], []
        for k in sel:
            A, Pm, cnt = py_momentum4((N, N, N), qi, qi[k])
            As.append(A)
            Ps.append(np.pad(Pm, ((0, len(qi) ** 2 - len(Pm)), (0, 0))))
            Cs.append(cnt)
        out[f"enum4_N{N}_q0"] = np.array(sel, np.int32)
        out[f"enum4_N{N}_A"] = np.array(As)
        out[f"enum4_N{N}_P"] = np.array(Ps)
        out[f"enum4_N{N}_C"] = np.array(Cs, np.int64)
    # tetrahedron weights: random energies, with ties and boundary hits
    cases = []
    for k in range(400):
        M = list(rng.normal(0.0, 1.0, 4))
        if k % 5 == 1:
            M[2] = M[0]
        if k % 7 == 3:
            M[3] = M[1] = M[2]
        Mqs = float(rng.normal(0.0, 1.0))
        if k % 11 == 4:
            Mqs = sorted(M)[k % 4]
        F = list(rng.normal(0.0, 1.0, 4))
        cases.append((Mqs, M, F))
    for strict in (0, 1):
        res_e, res_g, res_I, res_M, res_F, res_p = [], [], [], [], [], []
        for Mqs, M, F in cases:
            e, g, I, Ms, Fs, perm = py_find_g_iver(Mqs, M, F, strict)
            res_e.append(e); res_g.append(g); res_I.append(I); res_M.append(Ms); res_F.append(Fs); res_p.append(perm)
        out[f"giver{strict}_e"] = np.array(res_e)
        out[f"giver{strict}_g"] = np.array(res_g)
        out[f"giver{strict}_I"] = np.array(res_I)
        out[f"giver{strict}_Ms"] = np.array(res_M)
        out[f"giver{strict}_Fs"] = np.array(res_F)
        out[f"giver{strict}_perm"] = np.array(res_p, np.int32)
    out["giver_Mqs"] = np.array([c[0] for c in cases])
    out["giver_M"] = np.array([c[1] for c in cases])
    out["giver_F"] = np.array([c[2] for c in cases])
    # V3 for a few pairs on the 4^3 mesh (q0 = irreducible point 2), inputs stored
    N = 4
    qi, qf, _ = py_make_tetrahedron((N, N, N), G)
    W, _ = S.point_group(cr)
    q0i = np.array([1, 0, 0], np.int32)
    q0f = (G / N) @ q0i
    allq = np.vstack([q0f[None, :], qf])
    ph = P.get_phonon(cr.latvec, cr.mass, cr.fc2_atm_num, cr.fc2_atm_indx, cr.fc2, allq, [300.0])
    A, Pm, cnt = py_momentum3((N, N, N), qi, q0i)
    idx = cr.fc3_atm_indx
    btyp = idx[:, :, 3]
    posr = np.einsum("ij,mnj->mni", cr.latvec, idx[:, :, :3].astype(float))
    rsm = 1.0 / np.sqrt(cr.mass)
    pairs = [0, 3, len(Pm) // 2]
    Ws = []
    for k in pairs:
        g1, g2 = Pm[k]
        q0chk = (True if all(q0i == 0) else False, all(qi[g1 - 1] == 0), all(qi[g2 - 1] == 0))
        phi = py_scatter_mat_el(qf[g1 - 1], qf[g2 - 1], q0chk, cr.nbasis, cr.fc3, cr.fc3_atm_num, btyp, posr, rsm,
                                ph["evec"][0], ph["evec"][g1], ph["evec"][g2])
        o0, o1, o2 = ph["onebyomega"][0], ph["onebyomega"][g1], ph["onebyomega"][g2]
        Wv = np.zeros((6, 6, 6))
        for s in range(6):
            for s1 in range(6):
                for s2 in range(6):
                    p = phi[s][s1][s2]
                    Wv[s, s1, s2] = (p.real * p.real + p.imag * p.imag) * (o0[s] * o1[s1] * o2[s2]) * (C.Sctr3THz2 / (N ** 3))
        Ws.append(Wv)
    out["v3_q0int"] = q0i
    out["v3_pairs"] = np.array([Pm[k] for k in pairs], np.int32)
    out["v3_W"] = np.array(Ws)
    out["v3_evec"] = ph["evec"]          # [0] = q0, [1:] = grid
    out["v3_onebyomega"] = ph["onebyomega"]
    out["v3_fc3"] = cr.fc3
    out["v3_fc3_num"] = cr.fc3_atm_num
    out["v3_fc3_idx"] = cr.fc3_atm_indx
    out["v3_latvec"] = cr.latvec
    out["v3_mass"] = cr.mass
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_small.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
