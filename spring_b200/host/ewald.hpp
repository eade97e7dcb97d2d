// Host side of the dipole-dipole (Ewald) term of the dynamical matrix: the parameters and the
// q-independent tables.  Header-only so that the device library (csrc/k_ewald.cu) and the host
// library (the CPU tests) compile the same code.
//
// Follows set_EwaldParam (src/Kappa/Src/EwaldParam.f90): DecideEwaldParameters, the R and G
// point sets of mesh_points(cell, mesh, .false., .true.) (CreateMesh_mod.f90:32-83 with
// fold_indx, IndxChng_mod.f90:85-107), ConstTerm and SumRule; and the q-independent parts of
// RealSpaceEW / CombineZStar (src/Kappa/Src/EwaldSum_mod.f90:37-108, 465-497).
//
// Layouts are the reference's Fortran arrays: eps(3,3) and eps_inv(3,3) column-major, Zstar(3,3,Nb),
// and every 3x3xNbxNb block C(beta, alpha, nu, mu) stored at beta + 3 alpha + 9 nu + 9 Nb mu.
#pragma once

#include <cmath>
#include <complex>
#include <string>
#include <vector>

namespace spring_ewald {

constexpr int MAX_NB = 8;  // the device kernel's limit (Ndof <= 24)
constexpr double PI = 3.141592653589793;
constexpr double CMP_PREC = 1.0e-8;

struct Setup {
    int nb = 0;
    double lmb = 0.0, det = 0.0, vol = 0.0;
    int gmesh[3] = {0, 0, 0}, rmesh[3] = {0, 0, 0};
    double eps[9] = {}, eps_inv[9] = {};
    std::vector<double> tau;    // [nb][3] Cartesian basis positions
    std::vector<double> zstar;  // Zstar(3,3,nb)
    std::vector<double> rpts;   // [NR][3]
    std::vector<double> gpts;   // [NG][3]
    // Real-space term with the Born charges folded in, times Lmb^3 / sqrt(det):
    //   HZ_R(b, a, nu, mu) = sum_{ap, bp} Z(ap, a, mu) Z(bp, b, nu) hab_R(bp, ap, nu, mu)   [NR][9 nb^2]
    std::vector<double> hz;
    // Constant part: -Z(CConst) - delta_{mu nu} CSumq0(b, a, mu), complex [9 nb^2][2]
    std::vector<double> cc;
    int nr() const { return (int)rpts.size() / 3; }
    int ng() const { return (int)gpts.size() / 3; }
};

inline int ent(int nb, int b, int a, int nu, int mu) { return b + 3 * a + 9 * nu + 9 * nb * mu; }

// mesh_points(cell_vec, mesh, div_cell = .false., ZeroCentered = .true.)
inline std::vector<double> mesh_points(const double cell[9], const int mesh[3]) {
    std::vector<double> out;
    for (int i1 = 0; i1 < mesh[0]; ++i1)
        for (int i2 = 0; i2 < mesh[1]; ++i2)
            for (int i3 = 0; i3 < mesh[2]; ++i3) {
                int f[3] = {i1, i2, i3};
                for (int k = 0; k < 3; ++k)
                    if (f[k] > mesh[k] / 2) f[k] -= mesh[k];
                for (int r = 0; r < 3; ++r)
                    out.push_back(cell[r] * f[0] + cell[r + 3] * f[1] + cell[r + 6] * f[2]);
            }
    return out;
}

// H_func (EwaldSum_mod.f90:258-283)
inline void h_func(double ld, double& h1, double& h2) {
    const double cerfn = std::erfc(ld);
    const double y2 = ld * ld, invy2 = 1.0 / y2, invy3 = invy2 / ld;
    const double pe = (2.0 / std::sqrt(PI)) * std::exp(-y2);
    h1 = (3.0 * invy3 * cerfn + pe * (3.0 * invy2 + 2.0)) * invy2;
    h2 = cerfn * invy3 + pe * invy2;
}

// hab(b, a) of one (R, mu, nu) term of RealSpaceEW, unscaled; false for the R = 0, mu = nu term.
inline bool real_term(const Setup& S, const double* R, int mu, int nu, double hab[9]) {
    if (std::fabs(R[0]) < CMP_PREC && std::fabs(R[1]) < CMP_PREC && std::fabs(R[2]) < CMP_PREC && mu == nu)
        return false;
    double dV[3], delV[3];
    for (int i = 0; i < 3; ++i) dV[i] = R[i] + S.tau[3 * nu + i] - S.tau[3 * mu + i];
    for (int j = 0; j < 3; ++j) delV[j] = dV[0] * S.eps_inv[0 + 3 * j] + dV[1] * S.eps_inv[1 + 3 * j] + dV[2] * S.eps_inv[2 + 3 * j];
    double DC = std::sqrt(delV[0] * dV[0] + delV[1] * dV[1] + delV[2] * dV[2]);
    for (int j = 0; j < 3; ++j) delV[j] *= S.lmb;
    DC *= S.lmb;
    double h1, h2;
    h_func(DC, h1, h2);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) hab[b + 3 * a] = delV[a] * delV[b] * h1 - S.eps_inv[b + 3 * a] * h2;
    return true;
}

// CombineZStar of one (nu, mu) block: out(b, a) = sum Z(ap, a, mu) Z(bp, b, nu) in(bp, ap)
template <class T>
inline void combine_block(const Setup& S, int mu, int nu, const T* in, T* out) {
    const double* Zm = S.zstar.data() + 9 * mu;
    const double* Zn = S.zstar.data() + 9 * nu;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            T s = T(0);
            for (int ap = 0; ap < 3; ++ap)
                for (int bp = 0; bp < 3; ++bp) s += Zm[ap + 3 * a] * Zn[bp + 3 * b] * in[bp + 3 * ap];
            out[b + 3 * a] = s;
        }
}

inline void inverse3(const double m[9], double out[9], double& det) {
    // column-major m(i,j) = m[i + 3j]
    auto M = [&](int i, int j) { return m[i + 3 * j]; };
    det = M(0, 0) * (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1)) - M(0, 1) * (M(1, 0) * M(2, 2) - M(1, 2) * M(2, 0)) +
          M(0, 2) * (M(1, 0) * M(2, 1) - M(1, 1) * M(2, 0));
    double c[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            c[i + 3 * j] = M(i1, j1) * M(i2, j2) - M(i1, j2) * M(i2, j1);  // cofactor
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[i + 3 * j] = c[j + 3 * i] / det;  // adjugate / det
}

// The whole setup.  latvec(3,3) column-major (column k = lattice vector k); tau_frac(3,nb)
// (atm_pos); eps(3,3) (dielec); zstar(3,3,nb) (BornZ).  decide != 0: Lmb and Gmesh from
// DecideEwaldParameters(prec_ew, sup_cell); else lmb and gmesh as given.  rmesh always as given.
inline int setup(const double latvec[9], int nb, const double* tau_frac, const double* eps, const double* zstar,
                 int decide, double prec_ew, double lmb, const int gmesh[3], const int rmesh[3], const int sup_cell[3],
                 Setup& S, std::string& err) {
    if (nb < 1 || nb > MAX_NB) {
        err = "dipole term: 1 to 8 basis atoms";
        return 1;
    }
    for (int k = 0; k < 3; ++k)
        if (rmesh[k] < 1 || (!decide && gmesh[k] < 1)) {
            err = "dipole term: Rmesh (and Gmesh without decide_EwParam) must be positive";
            return 1;
        }
    S = Setup();
    S.nb = nb;
    for (int i = 0; i < 9; ++i) S.eps[i] = eps[i];
    // eps_inv = transpose(inverse(transpose(eps))) = inverse(eps)
    inverse3(S.eps, S.eps_inv, S.det);
    if (!(S.det > 0.0)) {
        err = "dipole term: the dielectric tensor must have a positive determinant";
        return 1;
    }
    auto A = [&](int r, int k) { return latvec[r + 3 * k]; };
    auto cross = [](const double* x, const double* y, double* z) {
        z[0] = x[1] * y[2] - x[2] * y[1];
        z[1] = x[2] * y[0] - x[0] * y[2];
        z[2] = x[0] * y[1] - x[1] * y[0];
    };
    double c23[3];
    cross(latvec + 3, latvec + 6, c23);
    S.vol = std::fabs(latvec[0] * c23[0] + latvec[1] * c23[1] + latvec[2] * c23[2]);
    double G[9];  // G(:, i) = cross(a_i2, a_i3) 2 pi / vol (unit_mod.f90:193-203)
    for (int i = 0; i < 3; ++i) {
        double g[3];
        cross(latvec + 3 * ((i + 1) % 3), latvec + 3 * ((i + 2) % 3), g);
        for (int r = 0; r < 3; ++r) G[r + 3 * i] = g[r] * 2.0 * PI / S.vol;
    }
    S.tau.resize(3 * nb);
    for (int mu = 0; mu < nb; ++mu)
        for (int r = 0; r < 3; ++r)
            S.tau[3 * mu + r] = A(r, 0) * tau_frac[3 * mu] + A(r, 1) * tau_frac[3 * mu + 1] + A(r, 2) * tau_frac[3 * mu + 2];
    S.zstar.assign(zstar, zstar + 9 * nb);
    if (decide) {  // DecideEwaldParameters (EwaldParam.f90)
        if (!(prec_ew > 0.0 && prec_ew < 1.0)) {
            err = "dipole term: prec_Ew must lie in (0, 1)";
            return 1;
        }
        const double p = -std::log(prec_ew);
        const int ncut = sup_cell[0] / 2 + 1;  // Ncut(2:) = 0
        double rcut[3], delV[3];
        for (int r = 0; r < 3; ++r) rcut[r] = A(r, 0) * ncut;
        for (int j = 0; j < 3; ++j)
            delV[j] = rcut[0] * S.eps_inv[0 + 3 * j] + rcut[1] * S.eps_inv[1 + 3 * j] + rcut[2] * S.eps_inv[2 + 3 * j];
        const double D = std::sqrt(delV[0] * rcut[0] + delV[1] * rcut[1] + delV[2] * rcut[2]);
        S.lmb = std::sqrt(p) / D;
        const double normG = std::sqrt(G[0] * G[0] + G[1] * G[1] + G[2] * G[2]);
        const double kcut = 2.0 * p / (D * std::sqrt((S.eps[0] + S.eps[4] + S.eps[8]) / 3.0));
        const int nk = (int)std::ceil(kcut / normG);
        for (int k = 0; k < 3; ++k) S.gmesh[k] = 2 * nk + 1;
    } else {
        if (!(lmb > 0.0)) {
            err = "dipole term: Lmb must be > 0";
            return 1;
        }
        S.lmb = lmb;
        for (int k = 0; k < 3; ++k) S.gmesh[k] = gmesh[k];
    }
    for (int k = 0; k < 3; ++k) S.rmesh[k] = rmesh[k];
    S.rpts = mesh_points(latvec, S.rmesh);
    S.gpts = mesh_points(G, S.gmesh);
    const int E = 9 * nb * nb, NR = S.nr(), NG = S.ng();
    const double rscale = S.lmb * S.lmb * S.lmb / std::sqrt(S.det);
    // real-space table
    S.hz.assign((size_t)NR * E, 0.0);
    for (int r = 0; r < NR; ++r)
        for (int mu = 0; mu < nb; ++mu)
            for (int nu = 0; nu < nb; ++nu) {
                double hab[9], hz[9];
                if (!real_term(S, &S.rpts[3 * r], mu, nu, hab)) continue;
                for (int i = 0; i < 9; ++i) hab[i] *= rscale;
                combine_block(S, mu, nu, hab, hz);
                for (int i = 0; i < 9; ++i) S.hz[(size_t)r * E + ent(nb, 0, 0, nu, mu) + i] = hz[i];
            }
    // SumRule: Cq0 = CK(0) - CR(0) - CConst, CSumq0(b, a, mu) = sum_nu Z(Cq0)(b, a, nu, mu)
    using cd = std::complex<double>;
    std::vector<cd> cq0(E, cd(0.0, 0.0));
    for (int g = 0; g < NG; ++g) {  // KSpaceEW at q = 0
        const double* K = &S.gpts[3 * g];
        if (!(std::fabs(K[0]) > CMP_PREC || std::fabs(K[1]) > CMP_PREC || std::fabs(K[2]) > CMP_PREC)) continue;
        double eK[3];
        for (int j = 0; j < 3; ++j) eK[j] = K[0] * S.eps[0 + 3 * j] + K[1] * S.eps[1 + 3 * j] + K[2] * S.eps[2 + 3 * j];
        const double KeK = K[0] * eK[0] + K[1] * eK[1] + K[2] * eK[2];
        const double KG = std::exp(-KeK / (4.0 * S.lmb * S.lmb)) / KeK;
        for (int mu = 0; mu < nb; ++mu)
            for (int nu = 0; nu < nb; ++nu) {
                double kt = 0.0;
                for (int i = 0; i < 3; ++i) kt += K[i] * (S.tau[3 * mu + i] - S.tau[3 * nu + i]);
                const cd Kmn = KG * std::exp(cd(0.0, kt));
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) cq0[ent(nb, b, a, nu, mu)] += K[a] * K[b] * Kmn;
            }
    }
    for (int i = 0; i < E; ++i) cq0[i] *= 4.0 * PI / S.vol;
    std::vector<cd> cr(E, cd(0.0, 0.0));
    for (int r = 0; r < NR; ++r)  // RealSpaceEW at q = 0
        for (int mu = 0; mu < nb; ++mu)
            for (int nu = 0; nu < nb; ++nu) {
                double hab[9];
                if (!real_term(S, &S.rpts[3 * r], mu, nu, hab)) continue;
                for (int i = 0; i < 9; ++i) cr[ent(nb, 0, 0, nu, mu) + i] += hab[i];
            }
    const double cnst = 4.0 * S.lmb * S.lmb * S.lmb / (3.0 * std::sqrt(PI) * std::sqrt(S.det));
    std::vector<cd> cconst(E, cd(0.0, 0.0));
    for (int mu = 0; mu < nb; ++mu)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) cconst[ent(nb, b, a, mu, mu)] = S.eps_inv[b + 3 * a] * cnst;
    for (int i = 0; i < E; ++i) cq0[i] = cq0[i] - cr[i] * rscale - cconst[i];
    std::vector<cd> cq0z(E), cconz(E);
    for (int mu = 0; mu < nb; ++mu)
        for (int nu = 0; nu < nb; ++nu) {
            combine_block(S, mu, nu, &cq0[ent(nb, 0, 0, nu, mu)], &cq0z[ent(nb, 0, 0, nu, mu)]);
            combine_block(S, mu, nu, &cconst[ent(nb, 0, 0, nu, mu)], &cconz[ent(nb, 0, 0, nu, mu)]);
        }
    S.cc.assign(2 * (size_t)E, 0.0);
    for (int mu = 0; mu < nb; ++mu)
        for (int nu = 0; nu < nb; ++nu)
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    cd v = -cconz[ent(nb, b, a, nu, mu)];
                    if (nu == mu)
                        for (int n2 = 0; n2 < nb; ++n2) v -= cq0z[ent(nb, b, a, n2, mu)];
                    S.cc[2 * ent(nb, b, a, nu, mu)] = v.real();
                    S.cc[2 * ent(nb, b, a, nu, mu) + 1] = v.imag();
                }
    return 0;
}

}  // namespace spring_ewald
