// Oracle — TEST INFRASTRUCTURE ONLY.  A CPU FP64 restatement of the SPRING
// phonon-scattering path, written loop-for-loop after the reference Fortran so
// that the GPU library can be checked against it.  Only tests/, bench.py's CPU
// baseline leg and __graft_entry__.smoke() load this library; the product
// (spring_b200) never does.
//
// Parity status: the reference Fortran cannot be compiled in this environment
// (no Fortran compiler, no HDF5, no spglib), and the reference ships no golden
// vectors for this path.  The restatement is pinned by the reference's own
// in-code invariants (count identities on odd meshes, sum of tetrahedron
// weights, FindIrrQ grid identity) and by known-answer tests in tests/.
//
// Array conventions: every array is the flat memory of the reference's Fortran
// array (column-major); comments give the Fortran shape.  Indices stored in
// arrays are 1-based like the reference's.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

namespace {

const double PI = 4.0 * std::atan(1.0);
const double Onebysqrt2PI = 1.0 / std::sqrt(2.0 * PI);
const double zero_prec = 5.0e-5;
const double OnebySix = 0.16666666666666666;
const double Sctr3THz2 = 1.054571817 * (1.60217733 * 1.60217733) *
                         (6.02214076 * 6.02214076 * 6.02214076) * 1000000.0 * PI * 0.0625;

inline int imod(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }

// dot_product(modulo(v, mesh), mesh_mul) + 1   (1-based grid index)
inline int grid_index(const int v[3], const int mesh[3]) {
    return imod(v[0], mesh[0]) + mesh[0] * imod(v[1], mesh[1]) +
           mesh[0] * mesh[1] * imod(v[2], mesh[2]) + 1;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// make_tetrahedron  (src/Kappa/Src/TetrahedronQ_m.f90:56-221, fold_indx
// src/Kappa/Src/IndxChng_mod.f90:85-107, MapAwayFromBZboundary :110-135)
//   q_pnt_int(3,Nq) int, q_pnt(3,Nq) f64, tetrahedrons(4,6*Nq) int (1-based)
//   G: 3x3 column-major, G(:,i) is reciprocal vector i.
// Returns 0, or -1 when a vertex maps outside the grid (the reference stops).
int orc_make_tetrahedron(const int* mesh, const int* shift, const double* G, int zero_centered,
                         int* q_pnt_int, double* q_pnt, int* tetrahedrons) {
    const int box[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 0, 1}, {0, 1, 1},
                           {1, 0, 1}, {1, 1, 1}, {1, 1, 0}, {0, 1, 0}};
    const int nq = mesh[0] * mesh[1] * mesh[2];
    std::vector<char> uniq(nq, 1);
    double Ru[3][3];  // Recp_cell_unit(:, i) = G(:, i)/mesh(i)
    for (int i = 0; i < 3; ++i)
        for (int r = 0; r < 3; ++r) Ru[r][i] = G[r + 3 * i] / double(mesh[i]);
    int tcount = 0;
    for (int iz = 0; iz < mesh[2]; ++iz)
        for (int iy = 0; iy < mesh[1]; ++iy)
            for (int ix = 0; ix < mesh[0]; ++ix) {
                int indx[3] = {ix, iy, iz}, vt[3];
                for (int d = 0; d < 3; ++d) {
                    vt[d] = indx[d];
                    if (zero_centered && vt[d] > mesh[d] / 2) vt[d] -= mesh[d];
                }
                int bt[8];
                for (int v = 0; v < 8; ++v) {
                    int vert[3], vf[3];
                    for (int d = 0; d < 3; ++d) vert[d] = box[v][d] + vt[d];
                    for (int d = 0; d < 3; ++d) {
                        vf[d] = vert[d];
                        if (zero_centered) {
                            if (vf[d] > mesh[d] / 2) vf[d] -= mesh[d];
                        } else {
                            if (vf[d] == mesh[d]) vf[d] -= mesh[d];
                            else if (vf[d] > mesh[d]) return -1;
                        }
                    }
                    int g = grid_index(vf, mesh);
                    if (g > nq) return -1;
                    bt[v] = g;
                    if (uniq[g - 1]) {
                        for (int d = 0; d < 3; ++d) q_pnt_int[3 * (g - 1) + d] = vf[d];
                        for (int r = 0; r < 3; ++r) {
                            double s = 0.0;
                            for (int c = 0; c < 3; ++c) s += Ru[r][c] * (double(vf[c]) + double(shift[c]) * 0.5);
                            q_pnt[3 * (g - 1) + r] = s;
                        }
                        uniq[g - 1] = 0;
                    }
                }
                const int pat[6][4] = {{0, 1, 2, 3}, {2, 3, 4, 1}, {5, 3, 4, 1},
                                       {5, 3, 6, 1}, {6, 3, 7, 1}, {0, 3, 7, 1}};
                for (int t = 0; t < 6; ++t)
                    for (int v = 0; v < 4; ++v) tetrahedrons[4 * (tcount + t) + v] = bt[pat[t][v]];
                tcount += 6;
            }
    return 0;
}

// ---------------------------------------------------------------------------
// Irreducible q-points.  Restates spglib 1.16.5 spg_get_ir_reciprocal_mesh
// (called at src/Kappa/Src/TetrahedronQ_m.f90:261) for a Gamma-centred mesh:
// every grid point maps to the smallest grid index in its orbit under the
// reciprocal rotations W^T (and -W^T when time_rev != 0).  Then unique_sort
// (Helper_m.f90:510-545) and FindPositionAndMultiplicity (:548-594).
//   rot: nrot integer 3x3 matrices W, row-major (x' = W x on fractional coords)
//   map_out(Nq) 0-based representative; irr(3,Nq0) addresses; pos(Nq) 1-based;
//   mult(Nq0).  Returns Nq0.
int orc_irr_q(const int* mesh, int nrot, const int* rot, int time_rev,
              const int* q_pnt_int, int* map_out, int* irr_q_pnt_int, int* pos, int* mult) {
    const int nq = mesh[0] * mesh[1] * mesh[2];
    std::vector<int> map(nq);
    for (int i = 0; i < nq; ++i) {
        const int* a = q_pnt_int + 3 * i;
        int best = i;
        for (int s = 0; s < nrot; ++s) {
            const int* W = rot + 9 * s;
            for (int sg = 0; sg < (time_rev ? 2 : 1); ++sg) {
                int b[3];
                for (int r = 0; r < 3; ++r) {
                    // (W^T a)_r = sum_c W[c][r] a_c
                    b[r] = W[0 * 3 + r] * a[0] + W[1 * 3 + r] * a[1] + W[2 * 3 + r] * a[2];
                    if (sg) b[r] = -b[r];
                }
                int g = grid_index(b, mesh) - 1;
                if (g < best) best = g;
            }
        }
        map[i] = best;
    }
    // unique_sort: ascending distinct representatives
    std::vector<int> uniq(map);
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    const int nirr = int(uniq.size());
    for (int k = 0; k < nirr; ++k) {
        mult[k] = 0;
        for (int d = 0; d < 3; ++d) irr_q_pnt_int[3 * k + d] = q_pnt_int[3 * uniq[k] + d];
    }
    for (int i = 0; i < nq; ++i) {
        map_out[i] = map[i];
        int k = int(std::lower_bound(uniq.begin(), uniq.end(), map[i]) - uniq.begin());
        pos[i] = k + 1;
        mult[k] += 1;
    }
    return nirr;
}

// ---------------------------------------------------------------------------
// MomentumConsrv3rd (src/Kappa/Src/QuasiMomentumConsrv3rd_m.f90:13-158),
// CheckIfWithinBZ (:161-173), Permutation3rd (:176-240).  The count
// assertions (:148-153) are not applied; counts are returned instead.
//   q_pnt_int(3,Nq); Allq1q2(4,Nq); q1q2_permuted(2,Nq) (first npairs used)
//   counts[0] = q1q2_count (pairs), counts[1] = total_count.
void orc_momentum3(const int* mesh, const int* q_pnt_int, const int* q0_int, int* Allq1q2,
                   int* q1q2_permuted, int* counts) {
    const int nq = mesh[0] * mesh[1] * mesh[2];
    const int sgn[3] = {0, 1, -1};
    int G[27][3];
    int gc = 0;
    for (int c3 = 0; c3 < 3; ++c3)
        for (int c2 = 0; c2 < 3; ++c2)
            for (int c1 = 0; c1 < 3; ++c1) {
                G[gc][0] = sgn[c1] * mesh[0];
                G[gc][1] = sgn[c2] * mesh[1];
                G[gc][2] = sgn[c3] * mesh[2];
                ++gc;
            }
    const int bound[3] = {mesh[0] / 2, mesh[1] / 2, mesh[2] / 2};
    std::vector<char> covered(nq, 0);
    std::memset(Allq1q2, 0, sizeof(int) * 4 * nq);
    int cnt = 0, total = 0;
    for (int i1 = 1; i1 <= nq; ++i1) {
        const int* q1 = q_pnt_int + 3 * (i1 - 1);
        int g1 = grid_index(q1, mesh);
        if (covered[g1 - 1]) continue;
        bool found = false;
        int q2[3], g2 = 0;
        for (int iG = 0; iG < 27; ++iG) {
            for (int d = 0; d < 3; ++d) q2[d] = G[iG][d] - (q0_int[d] + q1[d]);
            g2 = grid_index(q2, mesh);
            bool within = true;
            for (int d = 0; d < 3; ++d)
                if (q2[d] > bound[d] || q2[d] < -bound[d]) within = false;
            if (within && g2 <= nq && g2 >= 1) { found = true; break; }
        }
        if (!found) continue;  // reference prints a warning
        ++cnt;
        int* a = Allq1q2 + 4 * (g1 - 1);
        a[0] = 1; a[1] = cnt; a[2] = g1; a[3] = g2;
        covered[g1 - 1] = 1;
        ++total;
        q1q2_permuted[2 * (cnt - 1)] = g1;
        q1q2_permuted[2 * (cnt - 1) + 1] = g2;
        // Permutation3rd: per = (2,1); flagged when the swapped integer vectors differ
        bool differ = (q1[0] != q2[0]) || (q1[1] != q2[1]) || (q1[2] != q2[2]);
        if (differ) {
            int* b = Allq1q2 + 4 * (g2 - 1);
            b[0] = 0; b[1] = cnt; b[2] = g2; b[3] = g1;
            covered[g2 - 1] = 1;
            ++total;
        }
    }
    counts[0] = cnt;
    counts[1] = total;
}

// ---------------------------------------------------------------------------
// MomentumConsrv4th (src/Kappa/Src/QuasiMomentumConsrv4th_m.f90:32-206) and
// Permutation4th (:224-312).  Allq1q2q3(3,Nq,Nq) Fortran = flat
// [q1][q2][3]; q1q2q3_permuted(3, cap).  Count assertions (:190-200) are not
// applied.  counts[0] = q1q2q3_count, counts[1] = total_count.
// Returns -1 when more than `cap` quartets would be written.
int orc_momentum4(const int* mesh, const int* q_pnt_int, const int* q0_int, int* Allq1q2q3,
                  int* q1q2q3_permuted, long long cap, long long* counts) {
    const int nq = mesh[0] * mesh[1] * mesh[2];
    const int sgn[3] = {0, 1, -1};
    int G[27][3];
    int gc = 0;
    for (int c3 = 0; c3 < 3; ++c3)
        for (int c2 = 0; c2 < 3; ++c2)
            for (int c1 = 0; c1 < 3; ++c1) {
                G[gc][0] = sgn[c1] * mesh[0];
                G[gc][1] = sgn[c2] * mesh[1];
                G[gc][2] = sgn[c3] * mesh[2];
                ++gc;
            }
    const int bound[3] = {mesh[0] / 2, mesh[1] / 2, mesh[2] / 2};
    const int per[5][3] = {{0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    std::vector<char> covered((size_t)nq * nq, 0);   // AlreadyCovered(q2, q1) -> [q1][q2]
    long long cnt = 0, total = 0;
    for (int i1 = 1; i1 <= nq; ++i1) {
        const int* q1 = q_pnt_int + 3 * (i1 - 1);
        int g1 = grid_index(q1, mesh);
        for (int i2 = 1; i2 <= nq; ++i2) {
            const int* q2 = q_pnt_int + 3 * (i2 - 1);
            int g2 = grid_index(q2, mesh);
            if (covered[(size_t)(g1 - 1) * nq + (g2 - 1)]) continue;
            bool found = false;
            int q3[3], g3 = 0;
            for (int iG = 0; iG < 27; ++iG) {
                for (int d = 0; d < 3; ++d) q3[d] = G[iG][d] - (q0_int[d] + q1[d] + q2[d]);
                g3 = grid_index(q3, mesh);
                bool within = true;
                for (int d = 0; d < 3; ++d)
                    if (q3[d] > bound[d] || q3[d] < -bound[d]) within = false;
                if (within && g3 <= nq && g3 >= 1) { found = true; break; }
            }
            if (!found) continue;
            if (cnt >= cap) return -1;
            ++cnt;
            int* a = Allq1q2q3 + 3 * ((size_t)(g1 - 1) * nq + (g2 - 1));
            a[0] = 0; a[1] = (int)cnt; a[2] = g3;
            covered[(size_t)(g1 - 1) * nq + (g2 - 1)] = 1;
            ++total;
            q1q2q3_permuted[3 * (cnt - 1)] = g1;
            q1q2q3_permuted[3 * (cnt - 1) + 1] = g2;
            q1q2q3_permuted[3 * (cnt - 1) + 2] = g3;
            // Permutation4th
            const int* ini[3] = {q1, q2, q3};
            const int gi[3] = {g1, g2, g3};
            int pg[5][3];
            for (int pp = 0; pp < 5; ++pp) {
                for (int k = 0; k < 3; ++k) pg[pp][k] = gi[per[pp][k]];
                bool nonew = true;
                for (int k = 0; k < 3; ++k)
                    for (int d = 0; d < 3; ++d)
                        if (ini[per[pp][k]][d] != ini[k][d]) nonew = false;
                for (int qq = 0; qq < pp; ++qq)
                    nonew = nonew || (pg[pp][0] == pg[qq][0] && pg[pp][1] == pg[qq][1] && pg[pp][2] == pg[qq][2]);
                if (!nonew) {
                    int* b = Allq1q2q3 + 3 * ((size_t)(pg[pp][0] - 1) * nq + (pg[pp][1] - 1));
                    b[0] = pp + 1; b[1] = (int)cnt; b[2] = pg[pp][2];
                    covered[(size_t)(pg[pp][0] - 1) * nq + (pg[pp][1] - 1)] = 1;
                    ++total;
                }
            }
        }
    }
    counts[0] = cnt;
    counts[1] = total;
    return 0;
}

// ---------------------------------------------------------------------------
// ScatterProbAllq1 (src/Kappa/Src/ThirdOrder_m.f90:41-166) with ScatterMatEl
// (:278-386, the reference's 9-deep loop order) and ScatterProbability
// (:389-439).
//   fc3: fC(3,3,3,Na3,Na3,Nb); atm_num(Nb); basis_typ(Na3,Nb) 1-based;
//   atm_pos_r(3,Na3,Nb); onebysqrtmass(Nb);
//   q_pnt(3,Nq); q_pnt_int(3,Nq); q0_int(3);
//   evec0(Ndof,Ndof) = Evec(:,:,i0) of the q0 set; oneby0(Ndof);
//   evec(Ndof,Ndof,Nq), oneby(Ndof,Nq) of the grid;
//   q1q2_permuted(2,npairs);  Sctrq1(Ndof,Ndof,Ndof,Nq) output (zeroed here).
void orc_scatter_w3(int nb, int na3, const int* atm_num, const int* basis_typ,
                    const double* atm_pos_r, const double* fc3, const double* onebysqrtmass,
                    int nq, const double* q_pnt, const int* q_pnt_int, const int* q0_int,
                    const double* evec0_ri, const double* oneby0, const double* evec_ri,
                    const double* oneby, int npairs, const int* q1q2_permuted, double* sctr) {
    const int ndof = 3 * nb;
    const size_t n3 = (size_t)ndof * ndof * ndof;
    const cplx* evec0 = reinterpret_cast<const cplx*>(evec0_ri);
    const cplx* evec = reinterpret_cast<const cplx*>(evec_ri);
    std::memset(sctr, 0, sizeof(double) * n3 * nq);
    const double mfac = Sctr3THz2 / double(nq);
    const bool g0 = q0_int[0] == 0 && q0_int[1] == 0 && q0_int[2] == 0;
#pragma omp parallel for schedule(dynamic, 4)
    for (int ip = 0; ip < npairs; ++ip) {
        const int g1 = q1q2_permuted[2 * ip], g2 = q1q2_permuted[2 * ip + 1];
        const int* q1i = q_pnt_int + 3 * (g1 - 1);
        const int* q2i = q_pnt_int + 3 * (g2 - 1);
        const double* q1 = q_pnt + 3 * (g1 - 1);
        const double* q2 = q_pnt + 3 * (g2 - 1);
        const cplx* e1 = evec + (size_t)(g1 - 1) * ndof * ndof;
        const cplx* e2 = evec + (size_t)(g2 - 1) * ndof * ndof;
        int strt[3] = {1, 1, 1};
        if (g0) strt[0] = 4;
        if (q1i[0] == 0 && q1i[1] == 0 && q1i[2] == 0) strt[1] = 4;
        if (q2i[0] == 0 && q2i[1] == 0 && q2i[2] == 0) strt[2] = 4;
        std::vector<cplx> phi(n3, cplx(0.0, 0.0));  // Phi_ss1s2(s2,s1,s)
        for (int mu = 1; mu <= nb; ++mu) {
            const int natm = atm_num[mu - 1];
            for (int N1 = 1; N1 <= natm; ++N1) {
                const int nu = basis_typ[(N1 - 1) + na3 * (mu - 1)];
                const double* R1 = atm_pos_r + 3 * ((N1 - 1) + na3 * (mu - 1));
                const double qr1 = q1[0] * R1[0] + q1[1] * R1[1] + q1[2] * R1[2];
                const cplx ex1(std::cos(qr1), std::sin(qr1));
                for (int N2 = 1; N2 <= natm; ++N2) {
                    const int eta = basis_typ[(N2 - 1) + na3 * (mu - 1)];
                    const double* R2 = atm_pos_r + 3 * ((N2 - 1) + na3 * (mu - 1));
                    const double qr2 = q2[0] * R2[0] + q2[1] * R2[1] + q2[2] * R2[2];
                    const cplx ex2(std::cos(qr2), std::sin(qr2));
                    const double mass_fac = onebysqrtmass[mu - 1] * onebysqrtmass[nu - 1] * onebysqrtmass[eta - 1];
                    const cplx exm = ex1 * ex2 * mass_fac;
                    for (int al = 1; al <= 3; ++al) {
                        const int r0 = 3 * (mu - 1) + al;
                        for (int s = strt[0]; s <= ndof; ++s) {
                            const cplx w0 = evec0[(r0 - 1) + ndof * (s - 1)];
                            for (int be = 1; be <= 3; ++be) {
                                const int r1 = 3 * (nu - 1) + be;
                                for (int s1 = strt[1]; s1 <= ndof; ++s1) {
                                    const cplx w1 = e1[(r1 - 1) + ndof * (s1 - 1)];
                                    for (int ga = 1; ga <= 3; ++ga) {
                                        const int r2 = 3 * (eta - 1) + ga;
                                        const size_t fi = (size_t)(ga - 1) + 3 * ((be - 1) + 3 * ((al - 1) +
                                                          3 * ((N2 - 1) + (size_t)na3 * ((N1 - 1) + (size_t)na3 * (mu - 1)))));
                                        const cplx pm = fc3[fi] * exm;
                                        for (int s2 = strt[2]; s2 <= ndof; ++s2) {
                                            const cplx w2 = e2[(r2 - 1) + ndof * (s2 - 1)];
                                            phi[(s2 - 1) + ndof * ((s1 - 1) + (size_t)ndof * (s - 1))] += pm * w0 * w1 * w2;
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
        // ScatterProbability
        const double* o0 = oneby0;
        const double* o1 = oneby + (size_t)(g1 - 1) * ndof;
        const double* o2 = oneby + (size_t)(g2 - 1) * ndof;
        double* W1 = sctr + (size_t)(g1 - 1) * n3;
        double* W2 = sctr + (size_t)(g2 - 1) * n3;
        std::vector<double> Wp(n3, 0.0), Wd(n3, 0.0);
        for (int s = strt[0]; s <= ndof; ++s)
            for (int s1 = strt[1]; s1 <= ndof; ++s1)
                for (int s2 = strt[2]; s2 <= ndof; ++s2) {
                    const cplx p = phi[(s2 - 1) + ndof * ((s1 - 1) + (size_t)ndof * (s - 1))];
                    const double abs2 = p.real() * p.real() + p.imag() * p.imag();
                    const double el = abs2 * (o0[s - 1] * o1[s1 - 1] * o2[s2 - 1]);
                    Wd[(s2 - 1) + ndof * ((s1 - 1) + (size_t)ndof * (s - 1))] = el * mfac;
                    Wp[(s1 - 1) + ndof * ((s2 - 1) + (size_t)ndof * (s - 1))] = el * mfac;
                }
        std::memcpy(W1, Wd.data(), sizeof(double) * n3);
        if (g1 != g2) std::memcpy(W2, Wp.data(), sizeof(double) * n3);
    }
}

// ---------------------------------------------------------------------------
// my_sort (src/Kappa/Src/TetrahedronIntegration_m.f90:18-90): ascending sort
// of the four vertex energies (dlasrt 'I'); equal values take the original
// vertices in their original order (first uncovered match).
static void my_sort(double* om, double* F, int* v1, int* v2) {
    double omc[4], Fc[4];
    int v1c[4], v2c[4];
    for (int i = 0; i < 4; ++i) { omc[i] = om[i]; Fc[i] = F[i]; v1c[i] = v1[i]; v2c[i] = v2[i]; }
    std::sort(om, om + 4);
    bool covered[4] = {false, false, false, false};
    for (int ii = 0; ii < 4; ++ii) {
        int act = -1;
        for (int k = 0; k < 4; ++k)
            if (!covered[k] && omc[k] == om[ii]) { act = k; break; }
        covered[act] = true;
        v1[ii] = v1c[act]; v2[ii] = v2c[act]; F[ii] = Fc[act];
    }
}

// FindgAndIver (TetrahedronIntegration_m.f90:93-218).  `strict` selects the
// case bounds of the LineWidth/kappa_iter copies (strict '<'/'>' at every
// bound, src/LineWidth/Src/TetrahedronIntegration_m.f90:113,133,169);
// kappa.x uses the non-strict form.
static bool find_g_iver(double Mqs, double* g, double* I, double* M, double* F, int* v1, int* v2,
                        int strict) {
    my_sort(M, F, v1, v2);
    bool c1, c2, c3;
    if (!strict) {
        c1 = (Mqs >= M[0]) && (Mqs < M[1]);
        c2 = (Mqs >= M[1]) && (Mqs < M[2]);
        c3 = (Mqs >= M[2]) && (Mqs <= M[3]);
    } else {
        c1 = (Mqs > M[0]) && (Mqs < M[1]);
        c2 = (Mqs > M[1]) && (Mqs < M[2]);
        c3 = (Mqs > M[2]) && (Mqs < M[3]);
    }
    if (c1) {
        *g = (3.0 * ((Mqs - M[0]) * (Mqs - M[0]))) / ((M[1] - M[0]) * (M[2] - M[0]) * (M[3] - M[0]));
        I[0] = (((Mqs - M[1]) / (M[0] - M[1])) + ((Mqs - M[2]) / (M[0] - M[2])) +
                ((Mqs - M[3]) / (M[0] - M[3]))) / 3.0;
        for (int v = 1; v < 4; ++v) I[v] = ((Mqs - M[0]) / (M[v] - M[0])) / 3.0;
        return true;
    } else if (c2) {
        const double gg = (3.0 / ((M[1] - M[2]) * (M[3] - M[0]))) *
                          ((((Mqs - M[0]) * (Mqs - M[2])) / (M[2] - M[0])) -
                           (((Mqs - M[1]) * (Mqs - M[3])) / (M[1] - M[3])));
        *g = gg;
        const double den = gg * (M[3] - M[0]);
        I[0] = (((Mqs - M[3]) / (M[0] - M[3])) / 3.0) +
               ((((Mqs - M[2]) / (M[0] - M[2])) * ((Mqs - M[0]) / (M[2] - M[0])) *
                 ((Mqs - M[2]) / (M[1] - M[2]))) / den);
        const double t1 = (Mqs - M[3]) / (M[1] - M[3]);
        I[1] = (((Mqs - M[2]) / (M[1] - M[2])) / 3.0) + (((t1 * t1) * ((Mqs - M[1]) / (M[2] - M[1]))) / den);
        const double t2 = (Mqs - M[0]) / (M[2] - M[0]);
        I[2] = (((Mqs - M[1]) / (M[2] - M[1])) / 3.0) + (((t2 * t2) * ((Mqs - M[2]) / (M[1] - M[2]))) / den);
        I[3] = (((Mqs - M[0]) / (M[3] - M[0])) / 3.0) +
               ((((Mqs - M[1]) / (M[3] - M[1])) * ((Mqs - M[3]) / (M[1] - M[3])) *
                 ((Mqs - M[1]) / (M[2] - M[1]))) / den);
        return true;
    } else if (c3) {
        *g = (3.0 * ((Mqs - M[3]) * (Mqs - M[3]))) / ((M[3] - M[0]) * (M[3] - M[1]) * (M[3] - M[2]));
        for (int v = 0; v < 3; ++v) I[v] = ((Mqs - M[3]) / (M[v] - M[3])) / 3.0;
        I[3] = (((Mqs - M[0]) / (M[3] - M[0])) + ((Mqs - M[1]) / (M[3] - M[1])) +
                ((Mqs - M[2]) / (M[3] - M[2]))) / 3.0;
        return true;
    }
    *g = 0.0;
    for (int v = 0; v < 4; ++v) I[v] = 0.0;
    return false;
}

static double iver_x_fver(const double* I, const double* F, bool enter) {
    double s = 0.0;
    if (enter)
        for (int v = 0; v < 4; ++v) s += I[v] * F[v];
    return OnebySix * s;
}

// Exposed for known-answer tests of the tetrahedron weights.
int orc_find_g_iver(double Mqs, const double* M_in, const double* F_in, int strict, double* g_out,
                    double* I_out, double* M_sorted, double* F_sorted, int* perm) {
    double M[4], F[4];
    int v1[4] = {1, 2, 3, 4}, v2[4] = {1, 2, 3, 4};
    for (int i = 0; i < 4; ++i) { M[i] = M_in[i]; F[i] = F_in[i]; }
    bool e = find_g_iver(Mqs, g_out, I_out, M, F, v1, v2, strict);
    for (int i = 0; i < 4; ++i) { M_sorted[i] = M[i]; F_sorted[i] = F[i]; perm[i] = v1[i]; }
    return e ? 1 : 0;
}

// ---------------------------------------------------------------------------
// CalculateLwTetrahedron (src/Kappa/Src/ThirdOrder_m.f90:169-275) with
// FindFandOmegaAtVertices (TetrahedronIntegration_m.f90:259-295).
//   omega0(Ndof) of q0; omega(Ndof,Nq), nbe(Ndof,Nq) of the grid (one T);
//   sctr(Ndof,Ndof,Ndof,Nq); tetra(4,6Nq); Allq1q2(4,Nq); pol(2,3) 1-based.
//   lw(Ndof), P3_q0(Ndof), *P3.
void orc_lw3_tetra(int ndof, int nq, const double* omega0, const double* omega, const double* nbe,
                   const double* sctr, const int* tetra, const int* Allq1q2, const int* pol,
                   double* lw, double* P3_q0, double* P3) {
    const size_t n3 = (size_t)ndof * ndof * ndof;
    const int ntet = 6 * nq;
    for (int s = 0; s < ndof; ++s) { lw[s] = 0.0; P3_q0[s] = 0.0; }
    std::vector<double> p3s(ndof, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int s0 = pol[0]; s0 <= pol[1]; ++s0) {
        const double Mqs = omega0[s0 - 1];
        double lws = 0.0, p3 = 0.0;
        for (int nT = 0; nT < ntet; ++nT) {
            int tv1[4], tv2[4];
            for (int v = 0; v < 4; ++v) {
                tv1[v] = tetra[4 * nT + v];
                tv2[v] = Allq1q2[4 * (tv1[v] - 1) + 3];
            }
            for (int s1 = pol[2]; s1 <= pol[3]; ++s1)
                for (int s2 = pol[4]; s2 <= pol[5]; ++s2) {
                    double F1[4], F2[4], F3[4], M1[4], M2[4], M3[4];
                    for (int v = 0; v < 4; ++v) {
                        const int a = tv1[v] - 1, b = tv2[v] - 1;
                        const double W = sctr[(s2 - 1) + ndof * ((s1 - 1) + (size_t)ndof * (s0 - 1)) + n3 * a];
                        const double n1 = nbe[(s1 - 1) + (size_t)ndof * a];
                        const double n2 = nbe[(s2 - 1) + (size_t)ndof * b];
                        F1[v] = W * (n1 + n2 + 1.0);
                        F2[v] = W * (n1 - n2);
                        const double o1 = omega[(s1 - 1) + (size_t)ndof * a];
                        const double o2 = omega[(s2 - 1) + (size_t)ndof * b];
                        M1[v] = o1 + o2;
                        M2[v] = o2 - o1;
                        M3[v] = o1 - o2;
                    }
                    for (int v = 0; v < 4; ++v) F3[v] = F2[v];
                    double g, I[4];
                    int a1[4], a2[4];
                    bool e;
                    std::memcpy(a1, tv1, sizeof a1); std::memcpy(a2, tv2, sizeof a2);
                    e = find_g_iver(Mqs, &g, I, M1, F1, a1, a2, 0);
                    lws += g * iver_x_fver(I, F1, e); p3 += g;
                    std::memcpy(a1, tv1, sizeof a1); std::memcpy(a2, tv2, sizeof a2);
                    e = find_g_iver(Mqs, &g, I, M2, F2, a1, a2, 0);
                    lws += g * iver_x_fver(I, F2, e); p3 += g;
                    std::memcpy(a1, tv1, sizeof a1); std::memcpy(a2, tv2, sizeof a2);
                    e = find_g_iver(Mqs, &g, I, M3, F3, a1, a2, 0);
                    lws -= g * iver_x_fver(I, F3, e); p3 += g;
                }
        }
        lw[s0 - 1] = lws;
        P3_q0[s0 - 1] = p3;
    }
    double t = 0.0;
    for (int s = 0; s < ndof; ++s) t += P3_q0[s];
    *P3 = t;
}

// ---------------------------------------------------------------------------
// Gaussian linewidth: CalculateLinewidth (src/Kappa/Src/ThirdOrder_m.f90:442-543)
// with the branch start reset per q1 (the reference leaves strt(2)/strt(3) at 4
// after the first Gamma point, :483,500,509; W is zero for Gamma acoustic modes
// anyway, :413-437) and the polarisation window of CalculateLwTetrahedron.
//   Also returns the Gaussian phase space P3_q0(s0) = sum (d1+d2+d3).
void orc_lw3_gauss(int ndof, int nq, const double* omega0, const double* omega, const double* nbe,
                   const double* sctr, const int* Allq1q2, const int* q_pnt_int, const int* pol,
                   double sigma, double* lw, double* P3_q0) {
    const size_t n3 = (size_t)ndof * ndof * ndof;
    const double os = 1.0 / sigma, os2 = os * os;
    for (int s = 0; s < ndof; ++s) { lw[s] = 0.0; P3_q0[s] = 0.0; }
    // s0 outermost (parallel): for each s0 the q1 accumulation order is the reference's
#pragma omp parallel for schedule(static, 1)
    for (int s0 = pol[0]; s0 <= pol[1]; ++s0)
    for (int q1 = 0; q1 < nq; ++q1) {
        const int q2 = Allq1q2[4 * q1 + 3] - 1;
        const int* a = q_pnt_int + 3 * q1;
        const int* b = q_pnt_int + 3 * q2;
        const int st1 = (a[0] == 0 && a[1] == 0 && a[2] == 0) ? 4 : 1;
        const int st2 = (b[0] == 0 && b[1] == 0 && b[2] == 0) ? 4 : 1;
        {
            double acc = 0.0, ps = 0.0;
            for (int s1 = std::max(st1, pol[2]); s1 <= pol[3]; ++s1)
                for (int s2 = std::max(st2, pol[4]); s2 <= pol[5]; ++s2) {
                    const double o0 = omega0[s0 - 1];
                    const double o1 = omega[(s1 - 1) + (size_t)ndof * q1];
                    const double o2 = omega[(s2 - 1) + (size_t)ndof * q2];
                    const double n1 = nbe[(s1 - 1) + (size_t)ndof * q1];
                    const double n2 = nbe[(s2 - 1) + (size_t)ndof * q2];
                    const double d1 = o0 - o1 - o2, d2 = o0 + o1 - o2, d3 = o0 - o1 + o2;
                    const double e1 = os * Onebysqrt2PI * std::exp(-0.5 * os2 * (d1 * d1));
                    const double e2 = os * Onebysqrt2PI * std::exp(-0.5 * os2 * (d2 * d2));
                    const double e3 = os * Onebysqrt2PI * std::exp(-0.5 * os2 * (d3 * d3));
                    const double W = sctr[(s2 - 1) + ndof * ((s1 - 1) + (size_t)ndof * (s0 - 1)) + n3 * q1];
                    acc += W * (((n1 + n2 + 1.0) * e1) + ((n1 - n2) * (e2 - e3)));
                    ps += e1 + e2 + e3;
                }
            lw[s0 - 1] += acc;
            P3_q0[s0 - 1] += ps;
        }
    }
}

// ---------------------------------------------------------------------------
// CalculateIsoW (src/Kappa/Src/IsotopicScatter.f90:36-94):
//   W_iso(Ndof,Ndof,Nq) = (s1, s0, q1)
void orc_iso_w(int nb, int nq, const double* evec0_ri, const double* omega0, const double* evec_ri,
               const double* g2iso, double* w_iso) {
    const int ndof = 3 * nb;
    const cplx* e0 = reinterpret_cast<const cplx*>(evec0_ri);
    const cplx* ev = reinterpret_cast<const cplx*>(evec_ri);
#pragma omp parallel for
    for (int q1 = 0; q1 < nq; ++q1)
        for (int s0 = 0; s0 < ndof; ++s0) {
            const double M = omega0[s0];
            for (int s1 = 0; s1 < ndof; ++s1) {
                double acc = 0.0;
                for (int b = 0; b < nb; ++b) {
                    cplx d(0.0, 0.0);
                    for (int c = 0; c < 3; ++c)
                        d += std::conj(ev[(3 * b + c) + ndof * s1 + (size_t)ndof * ndof * q1]) * e0[(3 * b + c) + ndof * s0];
                    acc += g2iso[b] * (d.real() * d.real() + d.imag() * d.imag());
                }
                w_iso[s1 + ndof * s0 + (size_t)ndof * ndof * q1] = acc * PI * (M * M) * 0.5 / double(nq);
            }
        }
}

// CalculateIsoLwTetra (IsotopicScatter.f90:97-168): NaN g / I set to zero.
void orc_iso_lw_tetra(int ndof, int nq, const double* omega0, const double* omega, const double* w_iso,
                      const int* tetra, double* lw) {
    const int ntet = 6 * nq;
#pragma omp parallel for
    for (int s0 = 0; s0 < ndof; ++s0) {
        const double Mqs = omega0[s0];
        double acc = 0.0;
        for (int nT = 0; nT < ntet; ++nT) {
            const int* tv = tetra + 4 * nT;
            for (int s1 = 0; s1 < ndof; ++s1) {
                double F[4], M[4], I[4], g;
                int a1[4], a2[4];
                for (int v = 0; v < 4; ++v) {
                    const int q = tv[v] - 1;
                    F[v] = w_iso[s1 + ndof * s0 + (size_t)ndof * ndof * q];
                    M[v] = omega[s1 + (size_t)ndof * q];
                    a1[v] = a2[v] = tv[v];
                }
                bool e = find_g_iver(Mqs, &g, I, M, F, a1, a2, 0);
                for (int v = 0; v < 4; ++v) if (std::isnan(I[v])) I[v] = 0.0;
                if (std::isnan(g)) g = 0.0;
                acc += g * iver_x_fver(I, F, e);
            }
        }
        lw[s0] = acc;
    }
}

// Gaussian isotope scattering rate: sum_q1,s1 W_iso delta(omega0 - omega1)
// (build-side Gaussian form of CalculateIsoLwTetra; same units).
void orc_iso_lw_gauss(int ndof, int nq, const double* omega0, const double* omega, const double* w_iso,
                      double sigma, double* lw) {
    const double os = 1.0 / sigma, os2 = os * os;
    for (int s0 = 0; s0 < ndof; ++s0) {
        double acc = 0.0;
        for (int q = 0; q < nq; ++q)
            for (int s1 = 0; s1 < ndof; ++s1) {
                const double d = omega0[s0] - omega[s1 + (size_t)ndof * q];
                acc += w_iso[s1 + ndof * s0 + (size_t)ndof * ndof * q] * os * Onebysqrt2PI * std::exp(-0.5 * os2 * d * d);
            }
        lw[s0] = acc;
    }
}

// ---------------------------------------------------------------------------
// GrVelKronProdSymm (src/Kappa/Src/VelocityKronProd_symm.f90:34-91)
//   grp_vel(3,Ndof,Nq0); Rxyz(3,3,Nsym) column-major; mult(Nq0);
//   out KrnGrpVelSym(9,Ndof,Nq0) in kron_prod order (Helper_m.f90:670-697).
void orc_velkron_symm(int ndof, int nq0, const double* grp_vel, int nsym, const double* Rxyz,
                      const int* mult, double* krn) {
    for (int q = 0; q < nq0; ++q) {
        const double p = 1.0 / double(nsym / mult[q]);
        for (int s = 0; s < ndof; ++s) {
            const double* vg = grp_vel + 3 * (s + (size_t)ndof * q);
            double acc[9] = {0};
            for (int ns = 0; ns < nsym; ++ns) {
                const double* R = Rxyz + 9 * ns;
                double rv[3];
                for (int i = 0; i < 3; ++i) rv[i] = R[i] * vg[0] + R[i + 3] * vg[1] + R[i + 6] * vg[2];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) acc[3 * i + j] += rv[i] * rv[j];
            }
            for (int k = 0; k < 9; ++k) krn[k + 9 * (s + (size_t)ndof * q)] = acc[k] * p;
        }
    }
}

// kappa_noIter_symm (src/Kappa/Src/ThermalConductivity.f90:167-292):
//   sum over irreducible q0 with symmetrised v (x) v.  mode_k(9,Ndof) optional.
void orc_kappa_symm(int ndof, int nq, int nq0, const int* irr_q_pnt_int, const double* omega0,
                    const double* nbe0, const double* lw, const double* krn, int s_first, int s_last,
                    double vol, double T, double kw_m_k, double* kappa, double* mode_k) {
    const double f1 = kw_m_k / ((T * T) * vol);
    const double f2 = f1 / double(nq);
    for (int k = 0; k < 9; ++k) kappa[k] = 0.0;
    if (mode_k) for (int k = 0; k < 9 * ndof; ++k) mode_k[k] = 0.0;
    for (int q = 0; q < nq0; ++q) {
        const int* a = irr_q_pnt_int + 3 * q;
        int strt = s_first;
        if (a[0] == 0 && a[1] == 0 && a[2] == 0) strt = 4;
        for (int s = strt; s <= s_last; ++s) {
            const double om = omega0[(s - 1) + (size_t)ndof * q];
            const double n = nbe0[(s - 1) + (size_t)ndof * q];
            const double tau = 0.5 / lw[(s - 1) + (size_t)ndof * q];
            const double pre = (om * om) * n * (n + 1.0) * tau;
            for (int k = 0; k < 9; ++k) {
                const double kq = pre * krn[k + 9 * ((s - 1) + (size_t)ndof * q)];
                kappa[k] += kq;
                if (mode_k) mode_k[k + 9 * (s - 1)] += kq;
            }
        }
    }
    for (int k = 0; k < 9; ++k) kappa[k] *= f2;
    if (mode_k) for (int k = 0; k < 9 * ndof; ++k) mode_k[k] *= f2;
}

// kappa_noIter (ThermalConductivity.f90:36-164): full grid, v (x) v per q.
void orc_kappa_full(int ndof, int nq, const int* q_pnt_int, const int* pos, const double* omega,
                    const double* nbe, const double* grp_vel, const double* lw, int s_first, int s_last,
                    double vol, double T, double kw_m_k, double* kappa) {
    const double f1 = kw_m_k / ((T * T) * vol);
    const double f2 = f1 / double(nq);
    for (int k = 0; k < 9; ++k) kappa[k] = 0.0;
    for (int q = 0; q < nq; ++q) {
        const int* a = q_pnt_int + 3 * q;
        int strt = s_first;
        if (a[0] == 0 && a[1] == 0 && a[2] == 0) strt = 4;
        const int ip = pos[q] - 1;
        for (int s = strt; s <= s_last; ++s) {
            const double om = omega[(s - 1) + (size_t)ndof * q];
            const double n = nbe[(s - 1) + (size_t)ndof * q];
            const double* v = grp_vel + 3 * ((s - 1) + (size_t)ndof * q);
            const double tau = 0.5 / lw[(s - 1) + (size_t)ndof * ip];
            const double pre = (om * om) * n * (n + 1.0) * tau;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) kappa[3 * i + j] += pre * v[i] * v[j];
        }
    }
    for (int k = 0; k < 9; ++k) kappa[k] *= f2;
}

// ---------------------------------------------------------------------------
// Four-phonon matrix elements.
// ScatterMatEl4 (src/Kappa/Src/FourthOrder_m.f90:286-422) in the reference loop
// order, for one quartet: Phi(s3,s2,s1,s) = sum FC4(d,c,b,a,N3,N2,N1,mu)
// e^{i q1.R1} e^{i q2.R2} e^{i q3.R3} m^-1/2(mu,nu,eta,ro) e0(mu a,s) e1(nu b,s1) e2(eta c,s2) e3(ro d,s3),
// then ScatterProbability4 (:425-473): W = |Phi|^2 (1/w0)(1/w1)(1/w2)(1/w3) Sctr4THz2/Nq^2.
//   fc4(3,3,3,3,Na4,Na4,Na4,Nb); e*(Ndof,Ndof) [s][row] memory; q0chk = Gamma flags of q0..q3.
//   out W[s0][s1][s2][s3] (== Fortran W(s3,s2,s1,s0)).
static const double Sctr4THz2 = 0.125 * PI * ((1.054571817 * 1.602176565) * (1.054571817 * 1.602176565)) *
                                (6.022140857 * 6.022140857 * 6.022140857 * 6.022140857) * 1000000.0;

void orc_w4_naive(int nb, int na4, const int* atm_num, const int* basis_typ, const double* atm_pos_r,
                  const double* fc4, const double* onebysqrtmass, int nq, const double* q1, const double* q2,
                  const double* q3, const int* q0chk, const double* e0_ri, const double* o0, const double* e1_ri,
                  const double* o1, const double* e2_ri, const double* o2, const double* e3_ri, const double* o3,
                  double* W) {
    const int n = 3 * nb;
    const cplx* e0 = reinterpret_cast<const cplx*>(e0_ri);
    const cplx* e1 = reinterpret_cast<const cplx*>(e1_ri);
    const cplx* e2 = reinterpret_cast<const cplx*>(e2_ri);
    const cplx* e3 = reinterpret_cast<const cplx*>(e3_ri);
    const size_t n4 = (size_t)n * n * n * n;
    std::vector<cplx> phi(n4, cplx(0.0, 0.0));
    int strt[4];
    for (int k = 0; k < 4; ++k) strt[k] = q0chk[k] ? 3 : 0;
    for (int mu = 0; mu < nb; ++mu)
        for (int N1 = 0; N1 < atm_num[mu]; ++N1) {
            const int nu = basis_typ[N1 + na4 * mu] - 1;
            const double* R1 = atm_pos_r + 3 * (N1 + na4 * mu);
            const double a1 = q1[0] * R1[0] + q1[1] * R1[1] + q1[2] * R1[2];
            const cplx x1(std::cos(a1), std::sin(a1));
            for (int N2 = 0; N2 < atm_num[mu]; ++N2) {
                const int eta = basis_typ[N2 + na4 * mu] - 1;
                const double* R2 = atm_pos_r + 3 * (N2 + na4 * mu);
                const double a2 = q2[0] * R2[0] + q2[1] * R2[1] + q2[2] * R2[2];
                const cplx x2(std::cos(a2), std::sin(a2));
                for (int N3 = 0; N3 < atm_num[mu]; ++N3) {
                    const int ro = basis_typ[N3 + na4 * mu] - 1;
                    const double* R3 = atm_pos_r + 3 * (N3 + na4 * mu);
                    const double a3 = q3[0] * R3[0] + q3[1] * R3[1] + q3[2] * R3[2];
                    const cplx x3(std::cos(a3), std::sin(a3));
                    const double mf = onebysqrtmass[mu] * onebysqrtmass[nu] * onebysqrtmass[eta] * onebysqrtmass[ro];
                    const cplx em = mf * x1 * x2 * x3;
                    for (int al = 0; al < 3; ++al)
                        for (int s = strt[0]; s < n; ++s) {
                            const cplx w0 = e0[(3 * mu + al) + n * s];
                            for (int be = 0; be < 3; ++be)
                                for (int s1 = strt[1]; s1 < n; ++s1) {
                                    const cplx w1 = e1[(3 * nu + be) + n * s1];
                                    for (int ga = 0; ga < 3; ++ga)
                                        for (int s2 = strt[2]; s2 < n; ++s2) {
                                            const cplx w2 = e2[(3 * eta + ga) + n * s2];
                                            for (int de = 0; de < 3; ++de) {
                                                const size_t fi = de + 3 * (ga + 3 * (be + 3 * (al + 3 * (N3 + (size_t)na4 * (N2 + (size_t)na4 * (N1 + (size_t)na4 * mu))))));
                                                const cplx pm = fc4[fi] * em;
                                                for (int s3 = strt[3]; s3 < n; ++s3)
                                                    phi[((s * n + s1) * n + s2) * (size_t)n + s3] += pm * w0 * w1 * w2 * e3[(3 * ro + de) + n * s3];
                                            }
                                        }
                                }
                        }
                }
            }
        }
    const double mfac = Sctr4THz2 / (double(nq) * double(nq));
    for (int s = 0; s < n; ++s)
        for (int s1 = 0; s1 < n; ++s1)
            for (int s2 = 0; s2 < n; ++s2)
                for (int s3 = 0; s3 < n; ++s3) {
                    const size_t k = ((s * n + s1) * n + s2) * (size_t)n + s3;
                    const bool z = s < strt[0] || s1 < strt[1] || s2 < strt[2] || s3 < strt[3];
                    const double a2 = phi[k].real() * phi[k].real() + phi[k].imag() * phi[k].imag();
                    W[k] = z ? 0.0 : (a2 * (o0[s] * o1[s1] * o2[s2] * o3[s3])) * mfac;
                }
}

// The same W for many quartets with the sum regrouped (phases folded into FC4 per basis
// block, then four eigenvector contractions); OpenMP over quartets.
//   quartets(3,nquart) 1-based grid indices; q_pnt(3,Nq), q_pnt_int(3,Nq); q0 float/int;
//   evec grid (Ndof,Ndof,Nq), oneby grid; out W [quartet][s0][s1][s2][s3].
void orc_w4_factored(int nb, int na4, const int* atm_num, const int* basis_typ, const double* atm_pos_r,
                     const double* fc4, const double* onebysqrtmass, int nq, const double* q_pnt, const int* q_pnt_int,
                     const int* q0_int, const double* e0_ri, const double* o0, const double* evec_ri,
                     const double* oneby, long long nquart, const int* quart, double* Wout) {
    const int n = 3 * nb;
    const size_t n4 = (size_t)n * n * n * n;
    const cplx* e0 = reinterpret_cast<const cplx*>(e0_ri);
    const cplx* ev = reinterpret_cast<const cplx*>(evec_ri);
    const double mfac = Sctr4THz2 / (double(nq) * double(nq));
    const bool g0 = q0_int[0] == 0 && q0_int[1] == 0 && q0_int[2] == 0;
#pragma omp parallel
    {
        std::vector<cplx> D((size_t)3 * n * n * n), T1((size_t)3 * n * n * n), T2((size_t)3 * n * n * n),
            T3((size_t)3 * n * n * n), phi(n4);
#pragma omp for schedule(dynamic, 16)
        for (long long iq = 0; iq < nquart; ++iq) {
            const int g[3] = {quart[3 * iq] - 1, quart[3 * iq + 1] - 1, quart[3 * iq + 2] - 1};
            std::fill(phi.begin(), phi.end(), cplx(0.0, 0.0));
            for (int mu = 0; mu < nb; ++mu) {
                std::fill(D.begin(), D.end(), cplx(0.0, 0.0));
                std::vector<cplx> P[3];
                for (int k = 0; k < 3; ++k) {
                    P[k].resize(atm_num[mu]);
                    const double* q = q_pnt + 3 * g[k];
                    for (int N = 0; N < atm_num[mu]; ++N) {
                        const double* R = atm_pos_r + 3 * (N + na4 * mu);
                        const double a = q[0] * R[0] + q[1] * R[1] + q[2] * R[2];
                        const int b = basis_typ[N + na4 * mu] - 1;
                        P[k][N] = onebysqrtmass[b] * cplx(std::cos(a), std::sin(a));
                    }
                }
                // D[a][nu b][eta c][ro d]
                for (int N1 = 0; N1 < atm_num[mu]; ++N1)
                    for (int N2 = 0; N2 < atm_num[mu]; ++N2)
                        for (int N3 = 0; N3 < atm_num[mu]; ++N3) {
                            const int nu = basis_typ[N1 + na4 * mu] - 1, eta = basis_typ[N2 + na4 * mu] - 1,
                                      ro = basis_typ[N3 + na4 * mu] - 1;
                            const cplx ph = P[0][N1] * P[1][N2] * P[2][N3];
                            const double* f = fc4 + 81 * (N3 + (size_t)na4 * (N2 + (size_t)na4 * (N1 + (size_t)na4 * mu)));
                            for (int al = 0; al < 3; ++al)
                                for (int be = 0; be < 3; ++be)
                                    for (int ga = 0; ga < 3; ++ga)
                                        for (int de = 0; de < 3; ++de)
                                            D[((al * n + 3 * nu + be) * n + 3 * eta + ga) * n + 3 * ro + de] +=
                                                f[((al * 3 + be) * 3 + ga) * 3 + de] * ph;
                        }
                const cplx* e1 = ev + (size_t)g[0] * n * n;
                const cplx* e2 = ev + (size_t)g[1] * n * n;
                const cplx* e3 = ev + (size_t)g[2] * n * n;
                const size_t R3 = (size_t)3 * n * n;  // rows (a, nu b, eta c)
                for (size_t r = 0; r < R3; ++r)
                    for (int s3 = 0; s3 < n; ++s3) {
                        cplx acc(0.0, 0.0);
                        for (int k = 0; k < n; ++k) acc += D[r * n + k] * e3[k + n * s3];
                        T1[r * n + s3] = acc;
                    }
                // T2[a][nu b][s2][s3] = sum_{eta c} e2(eta c, s2) T1[a][nu b][eta c][s3]
                for (int ab = 0; ab < 3 * n; ++ab)
                    for (int s2 = 0; s2 < n; ++s2)
                        for (int s3 = 0; s3 < n; ++s3) {
                            cplx acc(0.0, 0.0);
                            for (int k = 0; k < n; ++k) acc += e2[k + n * s2] * T1[((size_t)ab * n + k) * n + s3];
                            T2[((size_t)ab * n + s2) * n + s3] = acc;
                        }
                // T3[a][s1][s2][s3] = sum_{nu b} e1(nu b, s1) T2[a][nu b][s2][s3]
                for (int a = 0; a < 3; ++a)
                    for (int s1 = 0; s1 < n; ++s1)
                        for (int s23 = 0; s23 < n * n; ++s23) {
                            cplx acc(0.0, 0.0);
                            for (int k = 0; k < n; ++k) acc += e1[k + n * s1] * T2[((size_t)a * n + k) * n * n + s23];
                            T3[((size_t)a * n + s1) * n * n + s23] = acc;
                        }
                for (int s = 0; s < n; ++s)
                    for (int a = 0; a < 3; ++a) {
                        const cplx w = onebysqrtmass[mu] * e0[(3 * mu + a) + n * s];
                        for (int k = 0; k < n * n * n; ++k) phi[(size_t)s * n * n * n + k] += w * T3[(size_t)a * n * n * n + k];
                    }
            }
            const bool gq[3] = {g[0] == 0, g[1] == 0, g[2] == 0};
            double* W = Wout + (size_t)iq * n4;
            const double* o1 = oneby + (size_t)g[0] * n;
            const double* o2 = oneby + (size_t)g[1] * n;
            const double* o3 = oneby + (size_t)g[2] * n;
            for (int s = 0; s < n; ++s)
                for (int s1 = 0; s1 < n; ++s1)
                    for (int s2 = 0; s2 < n; ++s2)
                        for (int s3 = 0; s3 < n; ++s3) {
                            const size_t k = ((s * n + s1) * n + s2) * (size_t)n + s3;
                            const bool z = (g0 && s < 3) || (gq[0] && s1 < 3) || (gq[1] && s2 < 3) || (gq[2] && s3 < 3);
                            const double a2 = phi[k].real() * phi[k].real() + phi[k].imag() * phi[k].imag();
                            W[k] = z ? 0.0 : (a2 * (o0[s] * o1[s1] * o2[s2] * o3[s3])) * mfac;
                        }
        }
    }
}

// TetrahedronIntegration4th / SumOverPolarization / FindFandOmegaVer_4th
// (src/Kappa/Src/Tetrahedron4th_sep.f90:37-425), one q0: for every q1 of the grid
// and every tetrahedron of q2, the vertices' q3, quartet number and permutation
// type come from Allq1q2q3 (as written by MomentumConsrv4th) and the W of a vertex
// is read from the stored quartet W with the reference's mode permutation
// (after_perm = before_perm(per(:, type))).  Three channels (1/6, 1/2, 1/2) with
// F divided by n0; NaN weights set to zero.
//   Allq1q2q3 [q1][q2][3]; Wq [quartet][s0][s1][s2][s3]; pol(2,4) 1-based;
//   omega0/nbe0 of q0 (Ndof); omega/nbe grid [q][s]; out rate(Ndof).
void orc_lw4_tetra(int ndof, int nq, const int* q0_int, const double* omega0, const double* nbe0, const double* omega,
                   const double* nbe, const int* tetra, const int* Allq1q2q3, const double* Wq, const int* pol,
                   double* rate) {
    const int n = ndof;
    const size_t n4 = (size_t)n * n * n * n;
    const int ntet = 6 * nq;
    const int per[5][3] = {{1, 3, 2}, {2, 1, 3}, {2, 3, 1}, {3, 1, 2}, {3, 2, 1}};
    const bool g0 = q0_int[0] == 0 && q0_int[1] == 0 && q0_int[2] == 0;
    const int s0a = g0 ? 4 : pol[0];
    std::vector<double> acc((size_t)n, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int s0 = s0a; s0 <= pol[1]; ++s0) {
        const double Mq0 = omega0[s0 - 1], n0 = nbe0[s0 - 1];
        double lw = 0.0;
        for (int q1 = 0; q1 < nq; ++q1) {
            for (int t = 0; t < ntet; ++t) {
                int v2[4], v3[4], typ[4], pos[4];
                for (int v = 0; v < 4; ++v) {
                    v2[v] = tetra[4 * t + v] - 1;
                    const int* e = Allq1q2q3 + 3 * ((size_t)q1 * nq + v2[v]);
                    typ[v] = e[0];
                    pos[v] = e[1] - 1;
                    v3[v] = e[2] - 1;
                }
                for (int s1 = pol[2]; s1 <= pol[3]; ++s1) {
                    const double M1s = omega[(size_t)q1 * n + s1 - 1], nq1 = nbe[(size_t)q1 * n + s1 - 1];
                    for (int s2 = pol[4]; s2 <= pol[5]; ++s2)
                        for (int s3 = pol[6]; s3 <= pol[7]; ++s3) {
                            double F1[4], F2[4], F3[4], M1[4], M2[4], M3[4];
                            const int before[3] = {s1, s2, s3};
                            for (int v = 0; v < 4; ++v) {
                                int after[3];
                                for (int k = 0; k < 3; ++k) after[k] = typ[v] == 0 ? before[k] : before[per[typ[v] - 1][k] - 1];
                                const double W = Wq[(size_t)pos[v] * n4 + (((size_t)(s0 - 1) * n + (after[0] - 1)) * n + (after[1] - 1)) * n + (after[2] - 1)];
                                const double n2 = nbe[(size_t)v2[v] * n + s2 - 1], n3 = nbe[(size_t)v3[v] * n + s3 - 1];
                                const double w2 = omega[(size_t)v2[v] * n + s2 - 1], w3 = omega[(size_t)v3[v] * n + s3 - 1];
                                F1[v] = W * (nq1 * n2 * n3 / n0);
                                M1[v] = (M1s + w2 + w3);
                                F2[v] = W * ((1.0 + nq1) * n2 * n3 / n0);
                                M2[v] = (w2 + w3 - M1s);
                                F3[v] = W * ((1.0 + nq1) * (1.0 + n2) * n3 / n0);
                                M3[v] = (w3 - M1s - w2);
                            }
                            double g, I[4];
                            int a1[4] = {0, 1, 2, 3}, a2[4] = {0, 1, 2, 3};
                            const double wts[3] = {OnebySix, 0.5, 0.5};
                            double* Fs[3] = {F1, F2, F3};
                            double* Ms[3] = {M1, M2, M3};
                            for (int ch = 0; ch < 3; ++ch) {
                                for (int v = 0; v < 4; ++v) { a1[v] = v; a2[v] = v; }
                                const bool e = find_g_iver(Mq0, &g, I, Ms[ch], Fs[ch], a1, a2, 0);
                                for (int v = 0; v < 4; ++v) if (std::isnan(I[v])) I[v] = 0.0;
                                if (std::isnan(g)) g = 0.0;
                                lw += wts[ch] * g * iver_x_fver(I, Fs[ch], e);
                            }
                        }
                }
            }
        }
        acc[s0 - 1] = lw;
    }
    for (int s = 0; s < n; ++s) rate[s] = acc[s];
}

// Gaussian form of the same rate (a build-side extension: the reference has only the
// tetrahedron form): sum over every grid (q1, q2) with q3 from the conservation law,
//   (1/6) F1 d(w0 - M1) + (1/2) F2 d(w0 - M2) + (1/2) F3 d(w0 - M3),
// with W computed directly for each ordered (q1, q2, q3) (no stored permutation).
//   W4 [q1][q2][s0][s1][s2][s3] for this q0 (from orc_w4_factored on every ordered pair).
void orc_lw4_gauss(int ndof, int nq, const int* q0_int, const double* omega0, const double* nbe0, const double* omega,
                   const double* nbe, const int* q3_of, const double* W4, const int* pol, double sigma, double* rate) {
    const int n = ndof;
    const size_t n4 = (size_t)n * n * n * n;
    const double os = 1.0 / sigma, os2 = os * os;
    const bool g0 = q0_int[0] == 0 && q0_int[1] == 0 && q0_int[2] == 0;
    const int s0a = g0 ? 4 : pol[0];
    for (int s = 0; s < n; ++s) rate[s] = 0.0;
#pragma omp parallel for schedule(dynamic, 1)
    for (int s0 = s0a; s0 <= pol[1]; ++s0) {
        const double w0 = omega0[s0 - 1], n0 = nbe0[s0 - 1];
        double lw = 0.0;
        for (int q1 = 0; q1 < nq; ++q1)
            for (int q2 = 0; q2 < nq; ++q2) {
                const int q3 = q3_of[(size_t)q1 * nq + q2];
                const double* W = W4 + ((size_t)q1 * nq + q2) * n4;
                for (int s1 = pol[2]; s1 <= pol[3]; ++s1) {
                    const double w1 = omega[(size_t)q1 * n + s1 - 1], n1 = nbe[(size_t)q1 * n + s1 - 1];
                    for (int s2 = pol[4]; s2 <= pol[5]; ++s2) {
                        const double w2 = omega[(size_t)q2 * n + s2 - 1], n2 = nbe[(size_t)q2 * n + s2 - 1];
                        for (int s3 = pol[6]; s3 <= pol[7]; ++s3) {
                            const double w3 = omega[(size_t)q3 * n + s3 - 1], n3 = nbe[(size_t)q3 * n + s3 - 1];
                            const double Wv = W[(((size_t)(s0 - 1) * n + s1 - 1) * n + s2 - 1) * n + s3 - 1];
                            const double d1 = w0 - (w1 + w2 + w3), d2 = w0 - (w2 + w3 - w1), d3 = w0 - (w3 - w1 - w2);
                            const double e1 = os * Onebysqrt2PI * std::exp(-0.5 * os2 * (d1 * d1));
                            const double e2 = os * Onebysqrt2PI * std::exp(-0.5 * os2 * (d2 * d2));
                            const double e3 = os * Onebysqrt2PI * std::exp(-0.5 * os2 * (d3 * d3));
                            lw += OnebySix * (Wv * (n1 * n2 * n3 / n0)) * e1 +
                                  0.5 * (Wv * ((1.0 + n1) * n2 * n3 / n0)) * e2 +
                                  0.5 * (Wv * ((1.0 + n1) * (1.0 + n2) * n3 / n0)) * e3;
                        }
                    }
                }
            }
        rate[s0 - 1] = lw;
    }
}

// ---------------------------------------------------------------------------
// Iterative BTE of kappa_iter.x (src/Kappa/Src_iterative):
//   TetrahedronWplus/Wminus (Quasi_momentum_consrv.f90:701-1208) -> 1/tau,
//   CreateFzero (HelperSubroutines.f90:118-185), TetrahedronIterPlus/Minus
//   (TetrahedronDeltaSum.f90:22-607), multiplyTaudFnew (:188-232), kappa (:277-347),
//   loop main.f90:295-361 (stop when max|dkappa| < eps_k or after max_iter).
// Irreducible set: time reversal only (q ~ -q), as Irr_q_point_m.f90:216-335.
// The W of each vertex is taken from kappa.x's Sctrq1 of the same q0 (both
// orientations of every pair are stored there), times 4: kappa_iter's
// Sctr3THz2 carries pi/4 where kappa.x's carries pi/16 (constants.f90:53-54).
// Vertex structure, in grid indices (0-based here):
//   plus  channel: vertex x, partner ConsrvPlus%q2indx = -p(x), M = w(-p(x),s2) - w(x,s1),
//                  W+ = 4 W3(q0; x s1; p(x) s2) (n(x,s1) - n(p(x),s2)),
//                  dF += (F(-p(x),s2) - F(x,s1)) terms;
//   minus channel: vertex v, partner u = q0 - v, M = w(v,s1) + w(u,s2),
//                  W- = 4 W3(q0; -v s1; p(-v) s2) (1 + n(-v,s1) + n(p(-v),s2)),
//                  dF += 0.5 (F(v,s1) + F(u,s2)) terms;
// where p(x) = grid(-q0 - x) is kappa.x's partner.  Strict case bounds, and a
// vertex set only counts when |sum(I) - 1| < zero_prec.
//   n_irr irreducible points: irr_grid[i] grid index of the representative,
//   pos_tr[q] irreducible index of grid point q, sgn_tr[q] = +1 (representative) / -1;
//   neg[q] grid index of -q; partner[i][q] = p(q) for q0 = irr i;
//   sctr[i][q][s0][s1][s2] kappa.x W3; omega[q][s], nbe[q][s] (one T), vel[q][s][3];
//   deg[i] number of grid points of irreducible point i.
// Outputs inv_tau[i][s], F[i][s][3], kappa_rta[9] (iteration 0), kappa[9]; returns iterations.
int orc_bte_iter(int ndof, int nq, const int* tetra, int n_irr, const int* irr_grid, const int* pos_tr,
                 const int* sgn_tr, const int* neg, const int* partner, const double* sctr, const double* omega,
                 const double* nbe, const double* vel, const int* deg, double T, double vol, double eps_k,
                 int max_iter, double* inv_tau, double* F, double* kappa_rta, double* kappa) {
    const int n = ndof;
    const size_t n3 = (size_t)n * n * n;
    const int ntet = 6 * nq;
    const double FunitE = 1.054571817 / 1.380649;
    const double kW_mK = 1.054571817 * 0.001;
    const double mfac_k = 1.0 / (double(nq) * vol);
    std::vector<double> F0((size_t)n_irr * n * 3, 0.0), dF((size_t)n_irr * n * 3, 0.0);
    auto Fat = [&](const double* Fv, int q, int s, int k) { return sgn_tr[q] * Fv[((size_t)pos_tr[q] * n + s) * 3 + k]; };

    // one pass over both channels; mode 0 accumulates 1/tau, mode 1 accumulates dF from Fv
    auto pass = [&](int mode, const double* Fv) {
#pragma omp parallel for schedule(dynamic, 1)
        for (int i = 0; i < n_irr; ++i) {
            const int g0 = irr_grid[i];
            const int* p = partner + (size_t)i * nq;
            const double* W3 = sctr + (size_t)i * nq * n3;
            for (int nT = 0; nT < ntet; ++nT) {
                int v1[4];
                for (int v = 0; v < 4; ++v) v1[v] = tetra[4 * nT + v] - 1;
                for (int s = 0; s < n; ++s) {
                    const double Mqs = omega[(size_t)g0 * n + s];
                    for (int s1 = 0; s1 < n; ++s1)
                        for (int s2 = 0; s2 < n; ++s2)
                            for (int ch = 0; ch < 2; ++ch) {
                                double M[4], Fdummy[4];
                                int a1[4], a2[4];
                                for (int v = 0; v < 4; ++v) {
                                    const int x = v1[v];
                                    if (ch == 0) {  // plus
                                        const int q2 = neg[p[x]];
                                        M[v] = omega[(size_t)q2 * n + s2] - omega[(size_t)x * n + s1];
                                        a2[v] = q2;
                                    } else {        // minus
                                        const int u = neg[p[neg[x]]];
                                        M[v] = omega[(size_t)x * n + s1] + omega[(size_t)u * n + s2];
                                        a2[v] = u;
                                    }
                                    a1[v] = x;
                                    Fdummy[v] = 0.0;
                                }
                                double g, I[4];
                                const bool e = find_g_iver(Mqs, &g, I, M, Fdummy, a1, a2, 1);
                                if (!e) continue;
                                const double sI = I[0] + I[1] + I[2] + I[3];
                                if (!(std::fabs(sI - 1.0) < zero_prec)) continue;
                                double tv = 0.0, tf[3] = {0.0, 0.0, 0.0};
                                for (int v = 0; v < 4; ++v) {
                                    const int x = a1[v];
                                    double Wv;
                                    if (ch == 0) {
                                        const double w3 = 4.0 * W3[(size_t)x * n3 + ((size_t)s * n + s1) * n + s2];
                                        Wv = w3 * (nbe[(size_t)x * n + s1] - nbe[(size_t)p[x] * n + s2]);
                                    } else {
                                        const int y = neg[x];
                                        const double w3 = 4.0 * W3[(size_t)y * n3 + ((size_t)s * n + s1) * n + s2];
                                        Wv = w3 * (1.0 + nbe[(size_t)y * n + s1] + nbe[(size_t)p[y] * n + s2]);
                                    }
                                    if (mode == 0) {
                                        tv += I[v] * Wv;
                                    } else {
                                        for (int k = 0; k < 3; ++k) {
                                            const double f1 = Fat(Fv, x, s1, k), f2 = Fat(Fv, a2[v], s2, k);
                                            tf[k] += (I[v] * Wv) * (ch == 0 ? (f2 - f1) : (f2 + f1));
                                        }
                                    }
                                }
                                const double pre = ch == 0 ? OnebySix * g : 0.5 * OnebySix * g;
                                if (mode == 0) inv_tau[(size_t)i * n + s] += pre * tv;
                                else
                                    for (int k = 0; k < 3; ++k) dF[((size_t)i * n + s) * 3 + k] += pre * tf[k];
                            }
                }
            }
        }
    };
    auto kappa_of = [&](const double* Fv, double* out) {
        for (int k = 0; k < 9; ++k) out[k] = 0.0;
        for (int i = 0; i < n_irr; ++i) {
            const int g0 = irr_grid[i];
            const bool gamma = g0 == 0;
            for (int s = gamma ? 3 : 0; s < n; ++s) {
                const double w = omega[(size_t)g0 * n + s], nq_ = nbe[(size_t)g0 * n + s];
                const double* v = vel + ((size_t)g0 * n + s) * 3;
                const double* f = Fv + ((size_t)i * n + s) * 3;
                const double pre = double(deg[i]) * w * nq_ * (nq_ + 1.0);
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) out[3 * a + b] += pre * (v[a] * f[b]);
            }
        }
        for (int k = 0; k < 9; ++k) out[k] = kW_mK * mfac_k * out[k];
    };

    for (size_t k = 0; k < (size_t)n_irr * n; ++k) inv_tau[k] = 0.0;
    pass(0, nullptr);
    for (int i = 0; i < n_irr; ++i) {
        const int g0 = irr_grid[i];
        for (int s = (g0 == 0 ? 3 : 0); s < n; ++s) {
            const double it = inv_tau[(size_t)i * n + s];
            if (std::fabs(it) > zero_prec)
                for (int k = 0; k < 3; ++k)
                    F0[((size_t)i * n + s) * 3 + k] =
                        FunitE * omega[(size_t)g0 * n + s] * vel[((size_t)g0 * n + s) * 3 + k] / (it * (T * T));
        }
    }
    std::vector<double> Fc(F0);
    kappa_of(Fc.data(), kappa_rta);
    double kold[9];
    for (int k = 0; k < 9; ++k) kold[k] = kappa_rta[k];
    int iter = 0;
    for (;;) {
        ++iter;
        std::fill(dF.begin(), dF.end(), 0.0);
        pass(1, Fc.data());
        for (int i = 0; i < n_irr; ++i) {
            const int g0 = irr_grid[i];
            for (int s = (g0 == 0 ? 3 : 0); s < n; ++s) {
                const double it = inv_tau[(size_t)i * n + s];
                if (std::fabs(it) > zero_prec)
                    for (int k = 0; k < 3; ++k) dF[((size_t)i * n + s) * 3 + k] /= it;
            }
        }
        for (size_t k = 0; k < Fc.size(); ++k) Fc[k] = F0[k] + dF[k];
        kappa_of(Fc.data(), kappa);
        double acc = 0.0;
        for (int k = 0; k < 9; ++k) acc = std::max(acc, std::fabs(kappa[k] - kold[k]));
        if (acc < eps_k || iter > max_iter) break;
        for (int k = 0; k < 9; ++k) kold[k] = kappa[k];
    }
    std::memcpy(F, Fc.data(), sizeof(double) * Fc.size());
    return iter;
}

// Iterative BTE with Gaussian delta weights (build-side form of kappa_iter.x; the reference's
// iterative solver integrates with tetrahedra only).  The same two channels and vertex structure as
// orc_bte_iter above, each grid point x taken once with the weight d(w0 - M) of a Gaussian of width
// sigma instead of the tetrahedron weights (the Gaussian form of kappa.x's linewidth, ThirdOrder_m.f90
// :521-533, applied to TetrahedronWplus/Wminus and TetrahedronIterPlus/Minus):
//   plus  at x:  M = w(-p(x),s2) - w(x,s1), W+ = 4 W3(q0; x s1; p(x) s2)(n(x,s1) - n(p(x),s2)),
//                1/tau += W+ d,   dF += W+ d (F(-p(x),s2) - F(x,s1));
//   minus at x:  u = -p(-x), M = w(x,s1) + w(u,s2), W- = 4 W3(q0; -x s1; p(-x) s2)(1 + n(-x,s1) + n(p(-x),s2)),
//                1/tau += 0.5 W- d, dF += 0.5 W- d (F(u,s2) + F(x,s1)).
// Arguments as orc_bte_iter, with sigma (rad/ps) in place of the tetrahedra.
int orc_bte_iter_gauss(int ndof, int nq, double sigma, int n_irr, const int* irr_grid, const int* pos_tr,
                       const int* sgn_tr, const int* neg, const int* partner, const double* sctr, const double* omega,
                       const double* nbe, const double* vel, const int* deg, double T, double vol, double eps_k,
                       int max_iter, double* inv_tau, double* F, double* kappa_rta, double* kappa) {
    const int n = ndof;
    const size_t n3 = (size_t)n * n * n;
    const double FunitE = 1.054571817 / 1.380649;
    const double kW_mK = 1.054571817 * 0.001;
    const double mfac_k = 1.0 / (double(nq) * vol);
    const double os = 1.0 / sigma, os2 = os * os;
    std::vector<double> F0((size_t)n_irr * n * 3, 0.0), dF((size_t)n_irr * n * 3, 0.0);
    auto Fat = [&](const double* Fv, int q, int s, int k) { return sgn_tr[q] * Fv[((size_t)pos_tr[q] * n + s) * 3 + k]; };
    auto delta = [&](double d) { return os * Onebysqrt2PI * std::exp(-0.5 * os2 * (d * d)); };
    auto pass = [&](int mode, const double* Fv) {
#pragma omp parallel for schedule(dynamic, 1)
        for (int i = 0; i < n_irr; ++i) {
            const int g0 = irr_grid[i];
            const int* p = partner + (size_t)i * nq;
            const double* W3 = sctr + (size_t)i * nq * n3;
            for (int s = 0; s < n; ++s) {
                const double w0 = omega[(size_t)g0 * n + s];
                double tv = 0.0, tf[3] = {0.0, 0.0, 0.0};
                for (int x = 0; x < nq; ++x)
                    for (int s1 = 0; s1 < n; ++s1)
                        for (int s2 = 0; s2 < n; ++s2) {
                            {  // plus
                                const int q2 = neg[p[x]];
                                const double M = omega[(size_t)q2 * n + s2] - omega[(size_t)x * n + s1];
                                const double w3 = 4.0 * W3[(size_t)x * n3 + ((size_t)s * n + s1) * n + s2];
                                const double Wv = w3 * (nbe[(size_t)x * n + s1] - nbe[(size_t)p[x] * n + s2]) * delta(w0 - M);
                                if (mode == 0) tv += Wv;
                                else
                                    for (int k = 0; k < 3; ++k) tf[k] += Wv * (Fat(Fv, q2, s2, k) - Fat(Fv, x, s1, k));
                            }
                            {  // minus
                                const int y = neg[x];
                                const int u = neg[p[y]];
                                const double M = omega[(size_t)x * n + s1] + omega[(size_t)u * n + s2];
                                const double w3 = 4.0 * W3[(size_t)y * n3 + ((size_t)s * n + s1) * n + s2];
                                const double Wv = 0.5 * w3 * (1.0 + nbe[(size_t)y * n + s1] + nbe[(size_t)p[y] * n + s2]) *
                                                  delta(w0 - M);
                                if (mode == 0) tv += Wv;
                                else
                                    for (int k = 0; k < 3; ++k) tf[k] += Wv * (Fat(Fv, u, s2, k) + Fat(Fv, x, s1, k));
                            }
                        }
                if (mode == 0) inv_tau[(size_t)i * n + s] = tv;
                else
                    for (int k = 0; k < 3; ++k) dF[((size_t)i * n + s) * 3 + k] = tf[k];
            }
        }
    };
    auto kappa_of = [&](const double* Fv, double* out) {
        for (int k = 0; k < 9; ++k) out[k] = 0.0;
        for (int i = 0; i < n_irr; ++i) {
            const int g0 = irr_grid[i];
            for (int s = (g0 == 0 ? 3 : 0); s < n; ++s) {
                const double w = omega[(size_t)g0 * n + s], nq_ = nbe[(size_t)g0 * n + s];
                const double* v = vel + ((size_t)g0 * n + s) * 3;
                const double* f = Fv + ((size_t)i * n + s) * 3;
                const double pre = double(deg[i]) * w * nq_ * (nq_ + 1.0);
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) out[3 * a + b] += pre * (v[a] * f[b]);
            }
        }
        for (int k = 0; k < 9; ++k) out[k] = kW_mK * mfac_k * out[k];
    };
    pass(0, nullptr);
    for (int i = 0; i < n_irr; ++i) {
        const int g0 = irr_grid[i];
        for (int s = (g0 == 0 ? 3 : 0); s < n; ++s) {
            const double it = inv_tau[(size_t)i * n + s];
            if (std::fabs(it) > zero_prec)
                for (int k = 0; k < 3; ++k)
                    F0[((size_t)i * n + s) * 3 + k] =
                        FunitE * omega[(size_t)g0 * n + s] * vel[((size_t)g0 * n + s) * 3 + k] / (it * (T * T));
        }
    }
    std::vector<double> Fc(F0);
    kappa_of(Fc.data(), kappa_rta);
    double kold[9];
    for (int k = 0; k < 9; ++k) kold[k] = kappa_rta[k];
    int iter = 0;
    for (;;) {
        ++iter;
        pass(1, Fc.data());
        for (int i = 0; i < n_irr; ++i) {
            const int g0 = irr_grid[i];
            for (int s = 0; s < n; ++s) {
                const double it = inv_tau[(size_t)i * n + s];
                const bool on = !(g0 == 0 && s < 3) && std::fabs(it) > zero_prec;
                for (int k = 0; k < 3; ++k) {
                    double& d = dF[((size_t)i * n + s) * 3 + k];
                    d = on ? d / it : d;
                }
            }
        }
        for (size_t k = 0; k < Fc.size(); ++k) Fc[k] = F0[k] + dF[k];
        kappa_of(Fc.data(), kappa);
        double acc = 0.0;
        for (int k = 0; k < 9; ++k) acc = std::max(acc, std::fabs(kappa[k] - kold[k]));
        if (acc < eps_k || iter > max_iter) break;
        for (int k = 0; k < 9; ++k) kold[k] = kappa[k];
    }
    std::memcpy(F, Fc.data(), sizeof(double) * Fc.size());
    return iter;
}

// ---------------------------------------------------------------------------
// Point-defect scattering: T-matrix with the tetrahedron Green's function
// (src/Kappa/Src/point_defect_m.f90:40-376, GreensFunc_m.f90:35-587).
// Energies are omega^2 in (rad/ps)^2 throughout, as ph_pd%omega and Wq0s02.

// my_sort_GF (GreensFunc_m.f90:80-150): ascending sort, vertex ids (and F) follow; equal values
// keep their original order (the first uncovered occurrence, as my_sort's cyclic search)
static void sort_gf(double* W, int* v, double* F) {
    double Wc[4], Fc[4] = {0, 0, 0, 0};
    int vc[4];
    for (int i = 0; i < 4; ++i) { Wc[i] = W[i]; vc[i] = v[i]; if (F) Fc[i] = F[i]; }
    std::sort(W, W + 4);
    bool covered[4] = {false, false, false, false};
    for (int ii = 0; ii < 4; ++ii) {
        int act = 0;
        for (int k = 0; k < 4; ++k)
            if (!covered[k] && Wc[k] == W[ii]) { act = k; break; }
        covered[act] = true;
        v[ii] = vc[act];
        if (F) F[ii] = Fc[act];
    }
}

static inline double sq(double x) { return x * x; }
static inline double cube(double x) { return x * x * x; }

// CoeffAtVerticesType0_1984 (:272-333): one pair (l, m) of equal vertex energies
static void coef_type0(const double* Wv, double W0, int l, int m, double* d) {
    int diff[2], c = 0;
    for (int v = 0; v < 4; ++v) if (v != l && v != m) diff[c++] = v;
    const int j = diff[0], k = diff[1];
    for (int v = 0; v < 4; ++v) d[v] = 0.0;
    const double Tjm = (W0 - Wv[j]) / (Wv[m] - Wv[j]);
    const double Tkm = (W0 - Wv[k]) / (Wv[m] - Wv[k]);
    const double dlm = (cube(W0 - Wv[j]) / ((Wv[j] - Wv[k]) * cube(Wv[j] - Wv[m]))) * std::log(std::fabs(W0 - Wv[j])) +
                       (cube(W0 - Wv[k]) / ((Wv[k] - Wv[j]) * cube(Wv[k] - Wv[m]))) * std::log(std::fabs(W0 - Wv[k])) +
                       ((W0 - Wv[m]) / ((Wv[m] - Wv[j]) * (Wv[m] - Wv[k]))) *
                           (0.5 + Tjm + Tkm + (Tjm * Tjm + Tkm * Tkm + Tjm * Tkm) * std::log(std::fabs(W0 - Wv[m])));
    d[l] = dlm;
    d[m] = dlm;
    for (int vv = 0; vv < 2; ++vv) {
        const int i = diff[vv], L = diff[(vv + 1) % 2];
        d[i] = (sq(W0 - Wv[i]) / (sq(Wv[i] - Wv[m]) * (Wv[L] - Wv[i]))) *
                   (1.0 + ((2.0 * (W0 - Wv[m]) / (Wv[i] - Wv[m])) + ((W0 - Wv[L]) / (Wv[i] - Wv[L]))) *
                              std::log(std::fabs(W0 - Wv[i]))) +
               (sq(W0 - Wv[m]) / (sq(Wv[m] - Wv[i]) * (Wv[L] - Wv[m]))) *
                   (1.0 + ((2.0 * (W0 - Wv[i]) / (Wv[m] - Wv[i])) + ((W0 - Wv[L]) / (Wv[m] - Wv[L]))) *
                              std::log(std::fabs(W0 - Wv[m]))) +
               (cube(W0 - Wv[L]) / (sq(Wv[L] - Wv[i]) * sq(Wv[L] - Wv[m]))) * std::log(std::fabs(W0 - Wv[L]));
    }
}

// CoeffAtVerticesType1_2004 (:336-371): vertices 1, 2, 3 equal
static void coef_type1(const double* Wv, double W0, double* d) {
    const double g1 = W0 - Wv[0], g4 = W0 - Wv[3];
    const double g41 = g4 / g1, g14 = g1 / g4;
    const double q = 11.0 / (6.0 * (1.0 - g41)) - 5.0 / (2.0 * sq(1.0 - g41)) + 1.0 / cube(1.0 - g41) +
                     std::log(std::fabs(g41)) / (sq(sq(1.0 - g14)) * g41);
    d[0] = d[1] = d[2] = q / g1;
    d[3] = (3.0 / sq(1.0 - g41) - 6.0 / cube(1.0 - g41) + 3.0 / sq(sq(1.0 - g41))) * (std::log(std::fabs(g14)) / g14) +
           1.0 / cube(1.0 - g14) + 2.5 * g41 / sq(1.0 - g41) - 2.0 * g41 / cube(1.0 - g41);
    d[3] = d[3] / g4;
}

// CoeffAtVerticesType3_2004 (:374-409): vertices 2, 3, 4 equal
static void coef_type3(const double* Wv, double W0, double* d) {
    const double g1 = W0 - Wv[0], g2 = W0 - Wv[1];
    const double g12 = g1 / g2, g21 = g2 / g1;
    const double q = 11.0 / (6.0 * (1.0 - g12)) - 5.0 / (2.0 * sq(1.0 - g12)) + 1.0 / cube(1.0 - g12) +
                     std::log(std::fabs(g12)) / (sq(sq(1.0 - g21)) * g12);
    d[1] = d[2] = d[3] = q / g2;
    d[0] = (3.0 / sq(1.0 - g12) - 6.0 / cube(1.0 - g12) + 3.0 / sq(sq(1.0 - g12))) * (std::log(std::fabs(g21)) / g21) +
           1.0 / cube(1.0 - g21) + 2.5 * g12 / sq(1.0 - g12) - 2.0 * g12 / cube(1.0 - g12);
    d[0] = d[0] / g1;
}

// CoeffAtVerticesType2_2004 (:412-447): vertices 1 = 2 and 3 = 4
static void coef_type2(const double* Wv, double W0, double* d) {
    const double g1 = W0 - Wv[0], g3 = W0 - Wv[2];
    const double g31 = g3 / g1, g13 = g1 / g3;
    const double q12 = 2.5 / sq(1.0 - g31) - 2.0 / cube(1.0 - g31) + g13 / cube(1.0 - g13) +
                       3.0 * (1.0 / cube(1.0 - g13) - 1.0 / sq(sq(1.0 - g13))) * (std::log(std::fabs(g31)) / g31);
    const double q34 = 2.5 / sq(1.0 - g13) - 2.0 / cube(1.0 - g13) + g31 / cube(1.0 - g31) +
                       3.0 * (1.0 / cube(1.0 - g31) - 1.0 / sq(sq(1.0 - g31))) * (std::log(std::fabs(g13)) / g13);
    d[0] = d[1] = q12 / g1;
    d[2] = d[3] = q34 / g3;
}

// CoeffAtVerticesTypeD_2004 (:450-496): all vertex energies distinct
static void coef_typeD(const double* Wv, double W0, double* d) {
    for (int v = 0; v < 4; ++v) {
        const double g1 = W0 - Wv[v], g2 = W0 - Wv[(v + 1) % 4], g3 = W0 - Wv[(v + 2) % 4], g4 = W0 - Wv[(v + 3) % 4];
        const double q = 1.0 / ((1.0 - g2 / g1) * (1.0 - g3 / g1) * (1.0 - g4 / g1)) +
                         (1.0 / (sq(1.0 - g1 / g2) * (1.0 - g3 / g2) * (1.0 - g4 / g2))) * (std::log(std::fabs(g2 / g1)) / (g2 / g1)) +
                         (1.0 / (sq(1.0 - g1 / g3) * (1.0 - g2 / g3) * (1.0 - g4 / g3))) * (std::log(std::fabs(g3 / g1)) / (g3 / g1)) +
                         (1.0 / (sq(1.0 - g1 / g4) * (1.0 - g2 / g4) * (1.0 - g3 / g4))) * (std::log(std::fabs(g4 / g1)) / (g4 / g1));
        d[v] = q / g1;
    }
}

// GFcoeffv_RealPart (:153-269): the degeneracy pattern of the sorted vertex energies picks the form
static void gf_real(const double* Wv, double W0, double* d) {
    bool check[4] = {true, true, true, true};
    int same = 0, types = 0, pairs[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    for (int i = 0; i < 4; ++i) {
        bool first = true;
        if (!check[i]) continue;
        for (int j = i + 1; j < 4; ++j)
            if (std::fabs(Wv[i] - Wv[j]) < zero_prec) {
                if (same < 3) { pairs[same][0] = i; pairs[same][1] = j; }
                ++same;
                if (first) { first = false; ++types; }
                check[j] = false;
            }
    }
    for (int v = 0; v < 4; ++v) d[v] = 0.0;
    if (same == 0) coef_typeD(Wv, W0, d);
    else if (same == 1) coef_type0(Wv, W0, pairs[0][0], pairs[0][1], d);
    else if (same == 2) {
        if (types == 1) {
            if (pairs[0][0] == 0 && pairs[1][0] == 0) coef_type1(Wv, W0, d);
            else if (pairs[0][0] == 1 && pairs[1][0] == 1) coef_type3(Wv, W0, d);
        } else if (types == 2) coef_type2(Wv, W0, d);
    } else if (same == 3) {
        for (int v = 0; v < 4; ++v) d[v] = 0.25 / (W0 - Wv[0]);
    }
}

// DiracDeltaCoeffVertices_1984 (:499-587), sorted energies E1..E4 and E
static void delta_coef(const double* Ev, double E, double* c) {
    const double E1 = Ev[0], E2 = Ev[1], E3 = Ev[2], E4 = Ev[3];
    const double cp = 1.0e-8;
    if ((E1 - E) <= cp && (E - E2) <= cp) {
        c[0] = ((E2 - E) / (E2 - E1) + (E3 - E) / (E3 - E1) + (E4 - E) / (E4 - E1)) *
               (sq(E - E1) / ((E4 - E1) * (E3 - E1) * (E2 - E1)));
        c[1] = cube(E - E1) / (sq(E2 - E1) * (E3 - E1) * (E4 - E1));
        c[2] = cube(E - E1) / ((E2 - E1) * sq(E3 - E1) * (E4 - E1));
        c[3] = cube(E - E1) / ((E2 - E1) * (E3 - E1) * sq(E4 - E1));
    } else if ((E2 - E) <= cp && (E - E3) <= cp) {
        const double a = ((E3 - E) * (E - E2)) / ((E4 - E2) * (E3 - E2)), b = ((E4 - E) * (E - E1)) / ((E4 - E1) * (E4 - E2)),
                     cc = ((E3 - E) * (E - E1)) / ((E3 - E2) * (E4 - E1));
        const double a2 = ((E4 - E) * (E - E1)) / ((E4 - E2) * (E3 - E1)), b2 = ((E4 - E) * (E - E2)) / ((E4 - E2) * (E3 - E2)),
                     c2 = ((E3 - E) * (E - E1)) / ((E3 - E1) * (E3 - E2));
        const double a3 = ((E3 - E) * (E - E2)) / ((E4 - E2) * (E3 - E1)), b3 = ((E4 - E) * (E - E2)) / ((E4 - E2) * (E4 - E1)),
                     c3 = ((E3 - E) * (E - E1)) / ((E3 - E1) * (E4 - E1));
        const double a4 = ((E3 - E) * (E - E2)) / ((E3 - E2) * (E3 - E1)), b4 = ((E4 - E) * (E - E1)) / ((E4 - E1) * (E3 - E1)),
                     c4 = ((E4 - E) * (E - E2)) / ((E3 - E2) * (E4 - E1));
        c[0] = ((E3 - E) / sq(E3 - E1)) * (a + b + cc) + ((E4 - E) / sq(E4 - E1)) * (a2 + b2 + c2);
        c[1] = ((E3 - E) / sq(E3 - E2)) * (a3 + b3 + c3) + ((E4 - E) / sq(E4 - E2)) * (a4 + b4 + c4);
        c[2] = ((E - E2) / sq(E3 - E2)) * (a3 + b3 + c3) + ((E - E1) / sq(E3 - E1)) * (a + b + cc);
        c[3] = ((E - E2) / sq(E4 - E2)) * (a4 + b4 + c4) + ((E - E1) / sq(E4 - E1)) * (a2 + b2 + c2);
        for (int v = 0; v < 4; ++v) c[v] *= 0.5;
    } else if ((E3 - E) <= cp && (E - E4) <= cp) {
        c[0] = cube(E4 - E) / (sq(E4 - E1) * (E4 - E2) * (E4 - E3));
        c[1] = cube(E4 - E) / ((E4 - E1) * sq(E4 - E2) * (E4 - E3));
        c[2] = cube(E4 - E) / ((E4 - E1) * (E4 - E2) * sq(E4 - E3));
        c[3] = ((E - E3) / (E4 - E3) + (E - E2) / (E4 - E2) + (E - E1) / (E4 - E1)) *
               (sq(E4 - E) / ((E4 - E1) * (E4 - E2) * (E4 - E3)));
    } else {
        for (int v = 0; v < 4; ++v) c[v] = 0.0;
    }
}

// CoefAtVertOfTetrhd (:35-77): sorts W (and v, F) in place; coefficient d - i pi c per sorted vertex,
// NaN parts set to zero.
void orc_pd_coeff(double W0, double* W, int* v, double* re, double* im) {
    sort_gf(W, v, nullptr);
    double d[4], c[4];
    gf_real(W, W0, d);
    delta_coef(W, W0, c);
    for (int k = 0; k < 4; ++k) {
        if (std::isnan(d[k])) d[k] = 0.0;
        if (std::isnan(c[k])) c[k] = 0.0;
        re[k] = d[k];
        im[k] = -PI * c[k];
    }
}

// PerturbationMatrix (point_defect_m.f90:40-108) and IFC2 (:111-136): home-cell FC2 blocks of the
// perturbed and pristine crystals (0 where the pair is absent).  V_FC(Ndof,Ndof) in (rad/ps)^2,
// V_M(Ndof,Ndof) diagonal (M_def - m) / m.
void orc_pd_perturbation(int nb, int na, const int* num, const int* idx, const double* fc, int na_p,
                         const int* num_p, const int* idx_p, const double* fc_p, const double* mass,
                         const double* mass_def, double* vfc, double* vm) {
    const int ndof = 3 * nb;
    const double wTHz = std::sqrt(1.60217733 * 6.02214076 * 10.0) * 10.0;
    auto ifc2 = [&](int nA, const int* nm, const int* ix, const double* f, int mu, int nu, int al, int be) {
        for (int N = 0; N < nm[mu]; ++N) {
            const int* e = ix + 4 * (N + nA * mu);
            if (e[3] - 1 == nu && e[0] == 0 && e[1] == 0 && e[2] == 0)
                return f[be + 3 * al + 9 * N + (size_t)9 * nA * mu];   // fC(1, beta, alpha, N, mu)
        }
        return 0.0;
    };
    for (int i = 0; i < ndof * ndof; ++i) { vfc[i] = 0.0; vm[i] = 0.0; }
    for (int nu = 0; nu < nb; ++nu)
        for (int be = 0; be < 3; ++be) {
            const int col = 3 * nu + be;
            for (int mu = 0; mu < nb; ++mu)
                for (int al = 0; al < 3; ++al) {
                    const int row = 3 * mu + al;
                    const double p = ifc2(na, num, idx, fc, mu, nu, al, be);
                    const double d = ifc2(na_p, num_p, idx_p, fc_p, mu, nu, al, be);
                    vfc[row + ndof * col] = (d - p) / std::sqrt(mass[mu] * mass[nu]) * (wTHz * wTHz);
                    if (mu == nu && al == be) vm[row + ndof * col] = (mass_def[mu] - mass[mu]) / mass[mu];
                }
        }
}

// zinverse (LAPACK zgetrf + zgetri): in place, false when a pivot is exactly zero
static bool cinverse(std::vector<cplx>& A, int n) {
    std::vector<int> piv(n);
    for (int k = 0; k < n; ++k) {  // LU with partial pivoting, column-major A(i, j) = A[i + n j]
        int p = k;
        for (int i = k + 1; i < n; ++i) if (std::abs(A[i + n * k]) > std::abs(A[p + n * k])) p = i;
        piv[k] = p;
        if (A[p + n * k] == cplx(0.0, 0.0)) return false;
        if (p != k) for (int j = 0; j < n; ++j) std::swap(A[k + n * j], A[p + n * j]);
        for (int i = k + 1; i < n; ++i) A[i + n * k] /= A[k + n * k];
        for (int j = k + 1; j < n; ++j)
            for (int i = k + 1; i < n; ++i) A[i + n * j] -= A[i + n * k] * A[k + n * j];
    }
    // inverse by solving A X = P I column by column
    std::vector<cplx> X((size_t)n * n, cplx(0.0, 0.0));
    for (int c = 0; c < n; ++c) {
        std::vector<cplx> b(n, cplx(0.0, 0.0));
        b[c] = 1.0;
        for (int k = 0; k < n; ++k) std::swap(b[k], b[piv[k]]);
        for (int i = 0; i < n; ++i) for (int j = 0; j < i; ++j) b[i] -= A[i + n * j] * b[j];
        for (int i = n - 1; i >= 0; --i) {
            for (int j = i + 1; j < n; ++j) b[i] -= A[i + n * j] * b[j];
            b[i] /= A[i + n * i];
        }
        for (int i = 0; i < n; ++i) X[i + n * c] = b[i];
    }
    A = X;
    return true;
}

// ScatterRatePointDefect (point_defect_m.f90:139-231) for one irreducible q0: tau_inv(Ndof).
// Point-defect mesh: tetra(4, 6 Nq) 1-based, w2(Ndof, Nq) = omega^2, evec(Ndof, Ndof, Nq)
// (Evec(row, s, q)); q0: omega0(Ndof) (rad/ps), e0(Ndof, Ndof); gamma0: q0 is Gamma.
void orc_pd_rate(int ndof, int nq, const int* tetra, const double* w2, const double* evec_ri,
                 const double* omega0, const double* e0_ri, int gamma0, const double* vfc, const double* vm,
                 double rho, double vol, int mat_inv_full, int optc_therm, double* tau_inv) {
    const cplx* ev = reinterpret_cast<const cplx*>(evec_ri);
    const cplx* e0 = reinterpret_cast<const cplx*>(e0_ri);
    const int n = ndof, ntet = 6 * nq;
    for (int s0 = 0; s0 < n; ++s0) tau_inv[s0] = 0.0;
    for (int s0 = gamma0 ? 3 : 0; s0 < n; ++s0) {
        const double W0 = omega0[s0] * omega0[s0];
        // GreensFunction: G = sum_tet sum_s sum_v Coeff_v F_v / NT, F_v = e e^H at the sorted vertex
        std::vector<cplx> G((size_t)n * n, cplx(0.0, 0.0));
        for (int t = 0; t < ntet; ++t)
            for (int s = 0; s < n; ++s) {
                double W[4], re[4], im[4];
                int v[4];
                for (int k = 0; k < 4; ++k) { v[k] = tetra[4 * t + k] - 1; W[k] = w2[s + (size_t)n * v[k]]; }
                orc_pd_coeff(W0, W, v, re, im);
                for (int k = 0; k < 4; ++k) {
                    const cplx cf(re[k], im[k]);
                    const cplx* e = ev + (size_t)n * s + (size_t)n * n * v[k];
                    for (int b = 0; b < n; ++b)
                        for (int a = 0; a < n; ++a) G[a + n * b] += cf * (e[a] * std::conj(e[b]));
                }
            }
        for (auto& g : G) g /= double(ntet);
        std::vector<double> V((size_t)n * n);
        for (int i = 0; i < n * n; ++i) V[i] = vfc[i] - W0 * vm[i];
        std::vector<cplx> VG((size_t)n * n, cplx(0.0, 0.0)), T((size_t)n * n, cplx(0.0, 0.0));
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k)
                for (int i = 0; i < n; ++i) VG[i + n * j] += V[i + n * k] * G[k + n * j];
        auto v_plus_vgv = [&]() {
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    cplx acc = V[i + n * j];
                    for (int k = 0; k < n; ++k) acc += VG[i + n * k] * V[k + n * j];
                    T[i + n * j] = acc;
                }
        };
        if (mat_inv_full) {
            std::vector<cplx> M((size_t)n * n);
            for (int i = 0; i < n * n; ++i) M[i] = -VG[i];
            for (int i = 0; i < n; ++i) M[i + n * i] += 1.0;
            if (!cinverse(M, n)) v_plus_vgv();
            else
                for (int j = 0; j < n; ++j)
                    for (int i = 0; i < n; ++i) {
                        cplx acc(0.0, 0.0);
                        for (int k = 0; k < n; ++k) acc += M[i + n * k] * V[k + n * j];
                        T[i + n * j] = acc;
                    }
        } else {
            v_plus_vgv();
        }
        const cplx* e = e0 + (size_t)n * s0;
        std::vector<cplx> Te(n, cplx(0.0, 0.0));
        for (int i = 0; i < n; ++i) for (int k = 0; k < n; ++k) Te[i] += T[i + n * k] * e[k];
        if (optc_therm) {
            cplx x(0.0, 0.0);
            for (int i = 0; i < n; ++i) x += std::conj(e[i]) * Te[i];
            tau_inv[s0] = rho * vol * (-x.imag() / omega0[s0]);
        } else {  // TetrahedronIntrg (:293-351)
            double acc = 0.0;
            for (int t = 0; t < ntet; ++t)
                for (int s = 0; s < n; ++s) {
                    double W[4], F[4], c[4];
                    int v[4];
                    for (int k = 0; k < 4; ++k) {
                        v[k] = tetra[4 * t + k] - 1;
                        W[k] = w2[s + (size_t)n * v[k]];
                        const cplx* eq = ev + (size_t)n * s + (size_t)n * n * v[k];
                        cplx d(0.0, 0.0);
                        for (int i = 0; i < n; ++i) d += std::conj(eq[i]) * Te[i];
                        F[k] = d.real() * d.real() + d.imag() * d.imag();
                    }
                    sort_gf(W, v, F);
                    delta_coef(W, W0, c);
                    for (int k = 0; k < 4; ++k) acc += c[k] * F[k];
                }
            tau_inv[s0] = rho * vol * (PI * acc / double(ntet)) / omega0[s0];
        }
    }
}

int orc_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}


// ---------------------------------------------------------------------------
// LineWidth.x path mode (src/LineWidth/Src/Linewidth_m.f90).
// ScatterMatEl (:500-591) + ScatterProbability (:594-657) for explicit
// (q1, q2) vectors: the 9-deep loop in the reference order, then
// W(s2,s1,s) = |Phi|^2 / (w0 w1 w2 Nq) * Sctr3THz2, zero below mode 4 where
// q0chk(k) is set.  q1v, q2v (n, 3); q0chk (n, 3) 0/1; e0 (Ndof x Ndof,
// Evec(row,s)); e1, e2 (n, Ndof x Ndof); w0 (Ndof); w1, w2 (n, Ndof);
// out W [pair][s0][s1][s2].
void orc_w3_path(int nb, int na3, const int* atm_num, const int* basis_typ, const double* atm_pos_r, const double* fc3,
                 const double* mass, int nq, int npairs, const double* q1v, const double* q2v, const int* q0chk,
                 const double* e0_ri, const double* w0, const double* e1_ri, const double* w1, const double* e2_ri,
                 const double* w2, double* Wout) {
    const int ndof = 3 * nb;
    const size_t n2 = (size_t)ndof * ndof, n3 = n2 * ndof;
    const cplx* evec0 = reinterpret_cast<const cplx*>(e0_ri);
#pragma omp parallel for schedule(dynamic, 1)
    for (int ip = 0; ip < npairs; ++ip) {
        const double* q1 = q1v + 3 * ip;
        const double* q2 = q2v + 3 * ip;
        const cplx* e1 = reinterpret_cast<const cplx*>(e1_ri) + ip * n2;
        const cplx* e2 = reinterpret_cast<const cplx*>(e2_ri) + ip * n2;
        int strt[3];
        for (int k = 0; k < 3; ++k) strt[k] = q0chk[3 * ip + k] ? 4 : 1;
        std::vector<cplx> phi(n3, cplx(0.0, 0.0));  // Phi_ss1s2(s2,s1,s)
        for (int mu = 1; mu <= nb; ++mu) {
            const int natm = atm_num[mu - 1];
            for (int N1 = 1; N1 <= natm; ++N1) {
                const int nu = basis_typ[(N1 - 1) + na3 * (mu - 1)];
                const double* R1 = atm_pos_r + 3 * ((N1 - 1) + na3 * (mu - 1));
                const double qr1 = q1[0] * R1[0] + q1[1] * R1[1] + q1[2] * R1[2];
                const cplx ex1(std::cos(qr1), std::sin(qr1));
                for (int N2 = 1; N2 <= natm; ++N2) {
                    const int eta = basis_typ[(N2 - 1) + na3 * (mu - 1)];
                    const double* R2 = atm_pos_r + 3 * ((N2 - 1) + na3 * (mu - 1));
                    const double qr2 = q2[0] * R2[0] + q2[1] * R2[1] + q2[2] * R2[2];
                    const cplx ex2(std::cos(qr2), std::sin(qr2));
                    const double mass_fac = 1.0 / std::sqrt(mass[mu - 1] * mass[nu - 1] * mass[eta - 1]);
                    const cplx exm = ex1 * ex2 * mass_fac;
                    for (int al = 1; al <= 3; ++al) {
                        const int r0 = 3 * (mu - 1) + al;
                        for (int s = strt[0]; s <= ndof; ++s) {
                            const cplx ww0 = evec0[(r0 - 1) + ndof * (s - 1)];
                            for (int be = 1; be <= 3; ++be) {
                                const int r1 = 3 * (nu - 1) + be;
                                for (int s1 = strt[1]; s1 <= ndof; ++s1) {
                                    const cplx ww1 = e1[(r1 - 1) + ndof * (s1 - 1)];
                                    for (int ga = 1; ga <= 3; ++ga) {
                                        const int r2 = 3 * (eta - 1) + ga;
                                        const size_t fi = (size_t)(ga - 1) + 3 * ((be - 1) + 3 * ((al - 1) +
                                                          3 * ((N2 - 1) + (size_t)na3 * ((N1 - 1) + (size_t)na3 * (mu - 1)))));
                                        const cplx pm = fc3[fi] * exm;
                                        for (int s2 = strt[2]; s2 <= ndof; ++s2) {
                                            const cplx ww2 = e2[(r2 - 1) + ndof * (s2 - 1)];
                                            phi[(s2 - 1) + ndof * ((s1 - 1) + (size_t)ndof * (s - 1))] += pm * ww0 * ww1 * ww2;
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
        double* W = Wout + (size_t)ip * n3;
        std::memset(W, 0, sizeof(double) * n3);
        const double* o1 = w1 + (size_t)ip * ndof;
        const double* o2 = w2 + (size_t)ip * ndof;
        for (int s = strt[0]; s <= ndof; ++s)
            for (int s1 = strt[1]; s1 <= ndof; ++s1)
                for (int s2 = strt[2]; s2 <= ndof; ++s2) {
                    const cplx p = phi[(s2 - 1) + ndof * ((s1 - 1) + (size_t)ndof * (s - 1))];
                    const double abs2 = p.real() * p.real() + p.imag() * p.imag();
                    const double el = abs2 / (w0[s - 1] * o1[s1 - 1] * o2[s2 - 1] * double(nq));
                    W[((size_t)(s - 1) * ndof + (s1 - 1)) * ndof + (s2 - 1)] = el * Sctr3THz2;
                }
    }
}

// CalculateLwTetrahedron of LineWidth.x (Linewidth_m.f90:326-417) with
// FindFandOmegaAtVertices (src/LineWidth/Src/TetrahedronIntegration_m.f90:257-293):
// the q2 phonons of vertex q1 come from its own table; strict case bounds.
//   omega0 (Ndof); omega1/nbe1 grid [q][s]; omega2/nbe2 [q1][s]; W [q1][s0][s1][s2];
//   tetra (6Nq, 4) 1-based; out lw (Ndof).
void orc_lw_path_tetra(int ndof, int nq, const double* omega0, const double* omega1, const double* nbe1,
                       const double* omega2, const double* nbe2, const double* W, const int* tetra, double* lw) {
    const int n = ndof;
    const size_t n3 = (size_t)n * n * n;
    const int ntet = 6 * nq;
#pragma omp parallel for schedule(dynamic, 1)
    for (int s0 = 1; s0 <= n; ++s0) {
        const double Mq0s = omega0[s0 - 1];
        double acc = 0.0;
        for (int t = 0; t < ntet; ++t) {
            int tv[4];
            for (int v = 0; v < 4; ++v) tv[v] = tetra[4 * t + v] - 1;
            for (int s1 = 1; s1 <= n; ++s1)
                for (int s2 = 1; s2 <= n; ++s2) {
                    double F1[4], F2[4], F3[4], M1[4], M2[4], M3[4];
                    for (int v = 0; v < 4; ++v) {
                        const int q = tv[v];
                        const double Wv = W[(size_t)q * n3 + ((size_t)(s0 - 1) * n + (s1 - 1)) * n + (s2 - 1)];
                        const double n1 = nbe1[(size_t)q * n + s1 - 1], n2 = nbe2[(size_t)q * n + s2 - 1];
                        const double o1 = omega1[(size_t)q * n + s1 - 1], o2 = omega2[(size_t)q * n + s2 - 1];
                        F1[v] = Wv * (n1 + n2 + 1.0);
                        F2[v] = Wv * (n1 - n2);
                        M1[v] = o1 + o2;
                        M2[v] = o2 - o1;
                        M3[v] = o1 - o2;
                    }
                    for (int v = 0; v < 4; ++v) F3[v] = F2[v];
                    double g, I[4];
                    int a1[4], a2[4];
                    for (int v = 0; v < 4; ++v) { a1[v] = v; a2[v] = v; }
                    bool e = find_g_iver(Mq0s, &g, I, M1, F1, a1, a2, 1);
                    acc += g * iver_x_fver(I, F1, e);
                    for (int v = 0; v < 4; ++v) { a1[v] = v; a2[v] = v; }
                    e = find_g_iver(Mq0s, &g, I, M2, F2, a1, a2, 1);
                    acc += g * iver_x_fver(I, F2, e);
                    for (int v = 0; v < 4; ++v) { a1[v] = v; a2[v] = v; }
                    e = find_g_iver(Mq0s, &g, I, M3, F3, a1, a2, 1);
                    acc -= g * iver_x_fver(I, F3, e);
                }
        }
        lw[s0 - 1] = acc;
    }
}

// CalculateLinewidth of LineWidth.x (Linewidth_m.f90:234-323) with the branch
// start reset for every q1 (the reference keeps strt(2)/strt(3) at 4 once set).
//   exists [q1]; q_pnt_int (Nq, 3); the rest as orc_lw_path_tetra.
void orc_lw_path_gauss(int ndof, int nq, const double* omega0, const double* omega1, const double* nbe1,
                       const double* omega2, const double* nbe2, const double* W, const int* exists,
                       const int* q_pnt_int, double sigma, double* lw) {
    const int n = ndof;
    const size_t n3 = (size_t)n * n * n;
    const double os = 1.0 / sigma, os2 = os * os;
    for (int s = 0; s < n; ++s) lw[s] = 0.0;
    for (int q1 = 0; q1 < nq; ++q1) {
        if (!exists[q1]) continue;
        const int* qi = q_pnt_int + 3 * q1;
        const int st1 = (qi[0] == 0 && qi[1] == 0 && qi[2] == 0) ? 4 : 1;
        const double* o2 = omega2 + (size_t)q1 * n;
        const int st2 = (std::fabs(o2[0]) < zero_prec && std::fabs(o2[1]) < zero_prec && std::fabs(o2[2]) < zero_prec) ? 4 : 1;
        for (int s0 = 1; s0 <= n; ++s0) {
            double t = 0.0;
            for (int s1 = st1; s1 <= n; ++s1)
                for (int s2 = st2; s2 <= n; ++s2) {
                    const double w1 = omega1[(size_t)q1 * n + s1 - 1], w2 = o2[s2 - 1];
                    const double n1 = nbe1[(size_t)q1 * n + s1 - 1], n2 = nbe2[(size_t)q1 * n + s2 - 1];
                    const double d1 = omega0[s0 - 1] - w1 - w2, d2 = omega0[s0 - 1] + w1 - w2, d3 = omega0[s0 - 1] - w1 + w2;
                    const double e1 = os * Onebysqrt2PI * std::exp(-0.5 * os2 * (d1 * d1));
                    const double e2 = os * Onebysqrt2PI * std::exp(-0.5 * os2 * (d2 * d2));
                    const double e3 = os * Onebysqrt2PI * std::exp(-0.5 * os2 * (d3 * d3));
                    t += W[(size_t)q1 * n3 + ((size_t)(s0 - 1) * n + (s1 - 1)) * n + (s2 - 1)] *
                         (((n1 + n2 + 1.0) * e1) + ((n1 - n2) * (e2 - e3)));
                }
            lw[s0 - 1] += t;
        }
    }
}

}  // extern "C"
