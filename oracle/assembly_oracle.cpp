// CPU restatement of the Blatter-Pattyn stiffness assembly -- TEST INFRASTRUCTURE ONLY.
//
// assemble_stiffness_matrix_3d (libglissade/glissade_velo_higher.F90:5382-5643) with the
// routines it calls, loop for loop and in the reference's operation order:
//   reference element, quadrature points and weights      glissade_velo_higher.F90:314-392
//   node shift tables ishift/jshift/kshift                  :455-478
//   get_basis_function_derivatives_3d                       :6508-6732
//   compute_effective_viscosity                             :7285-7470
//   compute_element_matrix                                  :8001-8123
//   element_to_global_matrix_3d                             :8200-8268
// check_symmetry_element_matrix (:10583-10644) only stops the run on an asymmetric element
// matrix; the element matrices here are symmetric by construction (each product is formed
// with the same operands in the same order on both sides of the diagonal, the factors 2 and 4
// scale exactly), so nothing is restated for it.  Fortran's x**2 is x*x; x**y with a real y is
// the C library's pow, as gfortran calls it.  Compiled -ffp-contract=off (no FMA).
//
// Arrays in the caller's Fortran layout (column-major, 1-based in the comments):
//   active_cell(nx,ny), xVertex/yVertex/stagusrf/stagthck(nx-1,ny-1), uvel/vvel(nz,nx-1,ny-1),
//   flwafact/efvs(nz-1,nx,ny), A**(27,nz,nx-1,ny-1).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <vector>

namespace {

constexpr int kApproxSIA = 0, kApproxSSA = 1;          // glide_types.F90:335-336 (else BP)
constexpr int kEfvsConstant = 0, kEfvsFlowfact = 1;    // glide_types.F90:240-242 (2: nonlinear)
constexpr double kVol0 = 1.0e9;                        // glissade_velo_higher.F90:1254
constexpr double kScyr = 31536000.0;                   // glimmer_physcon.F90:90
constexpr double kLenScale = 200.0e3;                  // glimmer_paramets.F90:97
constexpr double kVeloScale = 500.0 / kScyr;           // glimmer_paramets.F90:98

// ishift(7,n), jshift(7,n), kshift(7,n): node n of the element relative to node 7, whose
// (k,i,j) are the element's; ishift(nr,nc) = ishift(7,nc) - ishift(7,nr) and likewise.
constexpr int kIsh7[8] = {-1, 0, 0, -1, -1, 0, 0, -1};
constexpr int kJsh7[8] = {-1, -1, 0, 0, -1, -1, 0, 0};
constexpr int kKsh7[8] = {1, 1, 1, 1, 0, 0, 0, 0};

struct RefElement {
    double wqp[8];
    double dxr[8][8], dyr[8][8], dzr[8][8];  // [p][n]
    RefElement() {
        const double r = 1.0 / std::sqrt(3.0);
        const double xq[8] = {-r, r, r, -r, -r, r, r, -r};
        const double yq[8] = {-r, -r, r, r, -r, -r, r, r};
        const double zq[8] = {-r, -r, -r, -r, r, r, r, r};
        for (int p = 0; p < 8; ++p) {
            const double x = xq[p], y = yq[p], z = zq[p];
            wqp[p] = 1.0;
            dxr[p][0] = -(1.0 - y) * (1.0 - z) / 8.0;
            dxr[p][1] = (1.0 - y) * (1.0 - z) / 8.0;
            dxr[p][2] = (1.0 + y) * (1.0 - z) / 8.0;
            dxr[p][3] = -(1.0 + y) * (1.0 - z) / 8.0;
            dxr[p][4] = -(1.0 - y) * (1.0 + z) / 8.0;
            dxr[p][5] = (1.0 - y) * (1.0 + z) / 8.0;
            dxr[p][6] = (1.0 + y) * (1.0 + z) / 8.0;
            dxr[p][7] = -(1.0 + y) * (1.0 + z) / 8.0;
            dyr[p][0] = -(1.0 - x) * (1.0 - z) / 8.0;
            dyr[p][1] = -(1.0 + x) * (1.0 - z) / 8.0;
            dyr[p][2] = (1.0 + x) * (1.0 - z) / 8.0;
            dyr[p][3] = (1.0 - x) * (1.0 - z) / 8.0;
            dyr[p][4] = -(1.0 - x) * (1.0 + z) / 8.0;
            dyr[p][5] = -(1.0 + x) * (1.0 + z) / 8.0;
            dyr[p][6] = (1.0 + x) * (1.0 + z) / 8.0;
            dyr[p][7] = (1.0 - x) * (1.0 + z) / 8.0;
            dzr[p][0] = -(1.0 - x) * (1.0 - y) / 8.0;
            dzr[p][1] = -(1.0 + x) * (1.0 - y) / 8.0;
            dzr[p][2] = -(1.0 + x) * (1.0 + y) / 8.0;
            dzr[p][3] = -(1.0 - x) * (1.0 + y) / 8.0;
            dzr[p][4] = (1.0 - x) * (1.0 - y) / 8.0;
            dzr[p][5] = (1.0 + x) * (1.0 - y) / 8.0;
            dzr[p][6] = (1.0 + x) * (1.0 + y) / 8.0;
            dzr[p][7] = (1.0 - x) * (1.0 + y) / 8.0;
        }
    }
};

const RefElement &ref() {
    static const RefElement r;
    return r;
}

// get_basis_function_derivatives_3d (:6508-6732): Jacobian sums in node order, cofactors,
// detJ by the first row, Jinv = transpose(cofactor) / detJ, then dphi = Jinv * dphi_r.
// Returns false for a singular Jacobian (the reference stops with GM_FATAL).
bool basis_derivs_3d(const double *x, const double *y, const double *z, const double *dxr, const double *dyr,
                     const double *dzr, double *dx, double *dy, double *dz, double *detJ) {
    double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int n = 0; n < 8; ++n) {
        J[0][0] = J[0][0] + dxr[n] * x[n];
        J[0][1] = J[0][1] + dxr[n] * y[n];
        J[0][2] = J[0][2] + dxr[n] * z[n];
        J[1][0] = J[1][0] + dyr[n] * x[n];
        J[1][1] = J[1][1] + dyr[n] * y[n];
        J[1][2] = J[1][2] + dyr[n] * z[n];
        J[2][0] = J[2][0] + dzr[n] * x[n];
        J[2][1] = J[2][1] + dzr[n] * y[n];
        J[2][2] = J[2][2] + dzr[n] * z[n];
    }
    double c[3][3];
    c[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    c[0][1] = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]);
    c[0][2] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    c[1][0] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]);
    c[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
    c[1][2] = -(J[0][0] * J[2][1] - J[0][1] * J[2][0]);
    c[2][0] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    c[2][1] = -(J[0][0] * J[1][2] - J[0][2] * J[1][0]);
    c[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    const double det = J[0][0] * c[0][0] + J[0][1] * c[0][1] + J[0][2] * c[0][2];
    *detJ = det;
    if (!(std::fabs(det) > 0.0)) return false;
    double Ji[3][3];
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) Ji[row][col] = c[col][row] / det;
    for (int n = 0; n < 8; ++n) {
        dx[n] = Ji[0][0] * dxr[n] + Ji[0][1] * dyr[n] + Ji[0][2] * dzr[n];
        dy[n] = Ji[1][0] * dxr[n] + Ji[1][1] * dyr[n] + Ji[1][2] * dzr[n];
        dz[n] = Ji[2][0] * dxr[n] + Ji[2][1] * dyr[n] + Ji[2][2] * dzr[n];
    }
    return true;
}

// compute_effective_viscosity (:7285-7470) at one quadrature point of an 8-node element.
double efvs_qp(int whichefvs, int whichapprox, double efvs_constant, double effstrain_min, double n_glen,
               const double *dx, const double *dy, const double *dz, const double *u, const double *v,
               double flwafact) {
    const double p_effstr = (1.0 - n_glen) / n_glen;
    if (whichefvs == kEfvsConstant) return efvs_constant;
    if (whichefvs == kEfvsFlowfact) {
        const double effstrain = kVeloScale / kLenScale * kScyr;
        return flwafact * std::pow(effstrain, p_effstr);
    }
    double du_dx = 0.0, du_dy = 0.0, du_dz = 0.0, dv_dx = 0.0, dv_dy = 0.0, dv_dz = 0.0, sq;
    if (whichapprox == kApproxSIA) {
        for (int n = 0; n < 8; ++n) {
            du_dz = du_dz + dz[n] * u[n];
            dv_dz = dv_dz + dz[n] * v[n];
        }
        sq = effstrain_min * effstrain_min + 0.25 * (du_dz * du_dz + dv_dz * dv_dz);
    } else if (whichapprox == kApproxSSA) {
        for (int n = 0; n < 8; ++n) {
            du_dx = du_dx + dx[n] * u[n];
            du_dy = du_dy + dy[n] * u[n];
            dv_dx = dv_dx + dx[n] * v[n];
            dv_dy = dv_dy + dy[n] * v[n];
        }
        sq = effstrain_min * effstrain_min +
             (du_dx * du_dx + dv_dy * dv_dy + du_dx * dv_dy + 0.25 * ((dv_dx + du_dy) * (dv_dx + du_dy)));
    } else {
        for (int n = 0; n < 8; ++n) {
            du_dx = du_dx + dx[n] * u[n];
            du_dy = du_dy + dy[n] * u[n];
            du_dz = du_dz + dz[n] * u[n];
            dv_dx = dv_dx + dx[n] * v[n];
            dv_dy = dv_dy + dy[n] * v[n];
            dv_dz = dv_dz + dz[n] * v[n];
        }
        sq = effstrain_min * effstrain_min +
             (du_dx * du_dx + dv_dy * dv_dy + du_dx * dv_dy + 0.25 * ((dv_dx + du_dy) * (dv_dx + du_dy))) +
             0.25 * (du_dz * du_dz + dv_dz * dv_dz);
    }
    return flwafact * std::pow(sq, p_effstr / 2.0);
}

// compute_effective_viscosity (:7285-7470) for the SSA on a 4-node element (dphi_dz = 0).
double efvs_qp4(int whichefvs, double efvs_constant, double effstrain_min, double n_glen, const double *dx,
                const double *dy, const double *u, const double *v, double flwafact) {
    const double p_effstr = (1.0 - n_glen) / n_glen;
    if (whichefvs == kEfvsConstant) return efvs_constant;
    if (whichefvs == kEfvsFlowfact) return flwafact * std::pow(kVeloScale / kLenScale * kScyr, p_effstr);
    double du_dx = 0.0, du_dy = 0.0, dv_dx = 0.0, dv_dy = 0.0;
    for (int n = 0; n < 4; ++n) {
        du_dx = du_dx + dx[n] * u[n];
        du_dy = du_dy + dy[n] * u[n];
        dv_dx = dv_dx + dx[n] * v[n];
        dv_dy = dv_dy + dy[n] * v[n];
    }
    const double sq = effstrain_min * effstrain_min +
                      (du_dx * du_dx + dv_dy * dv_dy + du_dx * dv_dy + 0.25 * ((dv_dx + du_dy) * (dv_dx + du_dy)));
    return flwafact * std::pow(sq, p_effstr / 2.0);
}

// compute_element_matrix (:8001-8123): K += efvs*wqp*detJ/vol0 * (products), columns outer.
void element_matrix(int whichapprox, double wqp, double detJ, double efvs, const double *dx, const double *dy,
                    const double *dz, double Kuu[8][8], double Kuv[8][8], double Kvu[8][8], double Kvv[8][8]) {
    const double f = efvs * wqp * detJ / kVol0;
    for (int nc = 0; nc < 8; ++nc)
        for (int nr = 0; nr < 8; ++nr) {
            if (whichapprox == kApproxSIA) {
                Kuu[nr][nc] = Kuu[nr][nc] + f * (dz[nr] * dz[nc]);
                Kvv[nr][nc] = Kvv[nr][nc] + f * (dz[nr] * dz[nc]);
            } else if (whichapprox == kApproxSSA) {
                Kuu[nr][nc] = Kuu[nr][nc] + f * (4.0 * dx[nr] * dx[nc] + dy[nr] * dy[nc]);
                Kuv[nr][nc] = Kuv[nr][nc] + f * (2.0 * dx[nr] * dy[nc] + dy[nr] * dx[nc]);
                Kvu[nr][nc] = Kvu[nr][nc] + f * (2.0 * dy[nr] * dx[nc] + dx[nr] * dy[nc]);
                Kvv[nr][nc] = Kvv[nr][nc] + f * (4.0 * dy[nr] * dy[nc] + dx[nr] * dx[nc]);
            } else {
                Kuu[nr][nc] = Kuu[nr][nc] + f * (4.0 * dx[nr] * dx[nc] + dy[nr] * dy[nc] + dz[nr] * dz[nc]);
                Kuv[nr][nc] = Kuv[nr][nc] + f * (2.0 * dx[nr] * dy[nc] + dy[nr] * dx[nc]);
                Kvu[nr][nc] = Kvu[nr][nc] + f * (2.0 * dy[nr] * dx[nc] + dx[nr] * dy[nc]);
                Kvv[nr][nc] = Kvv[nr][nc] + f * (4.0 * dy[nr] * dy[nc] + dx[nr] * dx[nc] + dz[nr] * dz[nc]);
            }
        }
}

// The 2D reference element (glissade_velo_higher.F90:528-570): 4 Gauss points, weights 1.
struct RefElement2 {
    double phi[4][4], dxr[4][4], dyr[4][4];  // [p][n]
    RefElement2() {
        const double r = 1.0 / std::sqrt(3.0);
        const double xq[4] = {-r, r, r, -r};
        const double yq[4] = {-r, -r, r, r};
        for (int p = 0; p < 4; ++p) {
            const double x = xq[p], y = yq[p];
            phi[p][0] = (1.0 - x) * (1.0 - y) / 4.0;
            phi[p][1] = (1.0 + x) * (1.0 - y) / 4.0;
            phi[p][2] = (1.0 + x) * (1.0 + y) / 4.0;
            phi[p][3] = (1.0 - x) * (1.0 + y) / 4.0;
            dxr[p][0] = -(1.0 - y) / 4.0;
            dxr[p][1] = (1.0 - y) / 4.0;
            dxr[p][2] = (1.0 + y) / 4.0;
            dxr[p][3] = -(1.0 + y) / 4.0;
            dyr[p][0] = -(1.0 - x) / 4.0;
            dyr[p][1] = -(1.0 + x) / 4.0;
            dyr[p][2] = (1.0 + x) / 4.0;
            dyr[p][3] = (1.0 - x) / 4.0;
        }
    }
};

const RefElement2 &ref2() {
    static const RefElement2 r;
    return r;
}

// get_basis_function_derivatives_2d (:6319-6504)
bool basis_derivs_2d(const double *x, const double *y, const double *dxr, const double *dyr, double *dx, double *dy,
                     double *detJ) {
    double J00 = 0.0, J01 = 0.0, J10 = 0.0, J11 = 0.0;
    for (int n = 0; n < 4; ++n) {
        J00 = J00 + dxr[n] * x[n];
        J01 = J01 + dxr[n] * y[n];
        J10 = J10 + dyr[n] * x[n];
        J11 = J11 + dyr[n] * y[n];
    }
    const double det = J00 * J11 - J01 * J10;
    *detJ = det;
    if (!(std::fabs(det) > 0.0)) return false;
    const double i00 = J11 / det, i01 = -J01 / det, i10 = -J10 / det, i11 = J00 / det;
    for (int n = 0; n < 4; ++n) {
        dx[n] = 0.0 + i00 * dxr[n] + i01 * dyr[n];
        dy[n] = 0.0 + i10 * dxr[n] + i11 * dyr[n];
    }
    return true;
}

// 2D node n of the element relative to the element's (i, j): ishift(3,n), jshift(3,n)
constexpr int kIsh3[4] = {-1, 0, 0, -1};
constexpr int kJsh3[4] = {-1, -1, 0, 0};

}  // namespace

extern "C" {

// assemble_stiffness_matrix_2d (:4961-5378), SSA branch: flwafact averaged over the layers
// (glissade_vertical_average, glissade_grid_operators.F90:1882-1946, no mask), then every active
// cell j = nhalo+1..ny-nhalo+1, i = nhalo+1..nx-nhalo+1: 4 quadrature points (basis derivatives,
// the SSA viscosity at the averaged flow factor, h at the point, the SSA element matrix with
// h*efvs), efvs(k,i,j) the mean over the points for every layer, and the scatter
// element_to_global_matrix_2d (:8127-8196) with the standard indxA_2d.  Arrays: uvel/vvel,
// xVertex, yVertex, stagusrf, stagthck (nx-1,ny-1); flwafact/efvs (nz-1,nx,ny);
// A** (nx-1,ny-1,9).  Returns 0, 1 (singular Jacobian) or 2 (nhalo < 2).
int oracle_assemble_stiffness_2d(int nx, int ny, int nz, int nhalo, const double *sigma, const int32_t *active_cell,
                                 const double *xVertex, const double *yVertex, const double *uvel,
                                 const double *vvel, const double *stagthck, const double *flwafact, int whichefvs,
                                 double efvs_constant, double effstrain_min, double n_glen, double *efvs, double *Auu,
                                 double *Auv, double *Avu, double *Avv) {
    if (nhalo < 2) return 2;
    const long NX = nx - 1, NY = ny - 1, NQ = NX * NY;
    const RefElement2 &R = ref2();
    std::memset(efvs, 0, sizeof(double) * (size_t)(nz - 1) * nx * ny);
    for (double *A : {Auu, Auv, Avu, Avv}) std::memset(A, 0, sizeof(double) * 9 * (size_t)NQ);
    std::vector<double> ff2((size_t)nx * ny, 0.0);
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            double &f = ff2[(i - 1) + (size_t)nx * (j - 1)];
            f = 0.0;
            for (int k = 1; k <= nz - 1; ++k)
                f = f + flwafact[(k - 1) + (size_t)(nz - 1) * ((i - 1) + (size_t)nx * (j - 1))] * (sigma[k] - sigma[k - 1]);
        }
    for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
        for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
            if (!active_cell[(i - 1) + (long)nx * (j - 1)]) continue;
            double Kuu[4][4] = {}, Kuv[4][4] = {}, Kvu[4][4] = {}, Kvv[4][4] = {};
            double x[4], y[4], u[4], v[4], h[4];
            for (int n = 0; n < 4; ++n) {
                const long q = (long)(i + kIsh3[n] - 1) + NX * (j + kJsh3[n] - 1);
                x[n] = xVertex[q];
                y[n] = yVertex[q];
                u[n] = uvel[q];
                v[n] = vvel[q];
                h[n] = stagthck[q];
            }
            const double ffc = ff2[(i - 1) + (size_t)nx * (j - 1)];
            double evert[4];
            for (int p = 0; p < 4; ++p) {
                double dx[4], dy[4], detJ;
                if (!basis_derivs_2d(x, y, R.dxr[p], R.dyr[p], dx, dy, &detJ)) return 1;
                evert[p] = efvs_qp4(whichefvs, efvs_constant, effstrain_min, n_glen, dx, dy, u, v, ffc);
                double h_qp = 0.0;
                for (int n = 0; n < 4; ++n) h_qp = h_qp + R.phi[p][n] * h[n];
                const double f = h_qp * evert[p] * 1.0 * detJ / kVol0;
                for (int nc = 0; nc < 4; ++nc)
                    for (int nr = 0; nr < 4; ++nr) {
                        Kuu[nr][nc] = Kuu[nr][nc] + f * (4.0 * dx[nr] * dx[nc] + dy[nr] * dy[nc]);
                        Kuv[nr][nc] = Kuv[nr][nc] + f * (2.0 * dx[nr] * dy[nc] + dy[nr] * dx[nc]);
                        Kvu[nr][nc] = Kvu[nr][nc] + f * (2.0 * dy[nr] * dx[nc] + dx[nr] * dy[nc]);
                        Kvv[nr][nc] = Kvv[nr][nc] + f * (4.0 * dy[nr] * dy[nc] + dx[nr] * dx[nc]);
                    }
            }
            for (int k = 1; k <= nz - 1; ++k) {
                double &e = efvs[(k - 1) + (long)(nz - 1) * ((i - 1) + (long)nx * (j - 1))];
                e = 0.0;
                for (int p = 0; p < 4; ++p) e = e + evert[p];
                e = e / 4;
            }
            for (int nr = 0; nr < 4; ++nr) {
                const long q = (long)(i + kIsh3[nr] - 1) + NX * (j + kJsh3[nr] - 1);
                for (int nc = 0; nc < 4; ++nc) {
                    const int m = (kIsh3[nc] - kIsh3[nr] + 1) + 3 * (kJsh3[nc] - kJsh3[nr] + 1);
                    const size_t a = (size_t)q + (size_t)NQ * m;
                    Auu[a] = Auu[a] + Kuu[nr][nc];
                    Auv[a] = Auv[a] + Kuv[nr][nc];
                    Avu[a] = Avu[a] + Kvu[nr][nc];
                    Avv[a] = Avv[a] + Kvv[nr][nc];
                }
            }
        }
    return 0;
}


// assemble_stiffness_matrix_3d (:5382-5643): efvs and A zeroed, then every active cell
// j = nhalo+1..ny-nhalo+1, i = nhalo+1..nx-nhalo+1 (j outer), element k = 1..nz-1: node
// coordinates, velocity, the eight quadrature points (basis derivatives, viscosity, element
// matrix), the mean viscosity, and the element matrix summed into A with the standard indxA_3d
// (m = 1 + (iA+1) + 3(jA+1) + 9(kA+1)).  Returns 0, or 1 for a singular Jacobian (A partly
// assembled, as far as the reference would have got before stopping), 2 for nhalo < 2 (element
// vertices outside the arrays).
int oracle_assemble_stiffness_3d(int nx, int ny, int nz, int nhalo, const double *sigma, const int32_t *active_cell,
                                 const double *xVertex, const double *yVertex, const double *uvel,
                                 const double *vvel, const double *stagusrf, const double *stagthck,
                                 const double *flwafact, int whichapprox, int whichefvs, double efvs_constant,
                                 double effstrain_min, double n_glen, double *efvs, double *Auu, double *Auv,
                                 double *Avu, double *Avv) {
    if (nhalo < 2) return 2;
    const long NX = nx - 1, NY = ny - 1;
    const RefElement &R = ref();
    std::memset(efvs, 0, sizeof(double) * (size_t)(nz - 1) * nx * ny);
    const size_t na = (size_t)27 * nz * NX * NY;
    for (double *A : {Auu, Auv, Avu, Avv}) std::memset(A, 0, sizeof(double) * na);
    auto V = [&](int i, int j) { return (long)(i - 1) + NX * (j - 1); };
    for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
        for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
            if (!active_cell[(i - 1) + (long)nx * (j - 1)]) continue;
            for (int k = 1; k <= nz - 1; ++k) {
                double Kuu[8][8] = {}, Kuv[8][8] = {}, Kvu[8][8] = {}, Kvv[8][8] = {};
                double x[8], y[8], z[8], u[8], v[8];
                for (int n = 0; n < 8; ++n) {
                    const int iN = i + kIsh7[n], jN = j + kJsh7[n], kN = k + kKsh7[n];
                    const long q = V(iN, jN);
                    x[n] = xVertex[q];
                    y[n] = yVertex[q];
                    z[n] = stagusrf[q] - sigma[kN - 1] * stagthck[q];
                    u[n] = uvel[(kN - 1) + (long)nz * q];
                    v[n] = vvel[(kN - 1) + (long)nz * q];
                }
                const double ff = flwafact[(k - 1) + (long)(nz - 1) * ((i - 1) + (long)nx * (j - 1))];
                double eq[8];
                for (int p = 0; p < 8; ++p) {
                    double dx[8], dy[8], dz[8], detJ;
                    if (!basis_derivs_3d(x, y, z, R.dxr[p], R.dyr[p], R.dzr[p], dx, dy, dz, &detJ)) return 1;
                    eq[p] = efvs_qp(whichefvs, whichapprox, efvs_constant, effstrain_min, n_glen, dx, dy, dz, u, v,
                                    ff);
                    element_matrix(whichapprox, R.wqp[p], detJ, eq[p], dx, dy, dz, Kuu, Kuv, Kvu, Kvv);
                }
                double &e = efvs[(k - 1) + (long)(nz - 1) * ((i - 1) + (long)nx * (j - 1))];
                e = 0.0;
                for (int p = 0; p < 8; ++p) e = e + eq[p];
                e = e / 8;
                // element_to_global_matrix_3d (:8200-8268)
                for (int nr = 0; nr < 8; ++nr) {
                    const int iR = i + kIsh7[nr], jR = j + kJsh7[nr], kR = k + kKsh7[nr];
                    for (int nc = 0; nc < 8; ++nc) {
                        const int kA = kKsh7[nc] - kKsh7[nr], iA = kIsh7[nc] - kIsh7[nr], jA = kJsh7[nc] - kJsh7[nr];
                        const int m = (iA + 1) + 3 * (jA + 1) + 9 * (kA + 1);
                        const size_t a = (size_t)m + 27 * ((size_t)(kR - 1) + (size_t)nz * (size_t)V(iR, jR));
                        Auu[a] = Auu[a] + Kuu[nr][nc];
                        Auv[a] = Auv[a] + Kuv[nr][nc];
                        Avu[a] = Avu[a] + Kvu[nr][nc];
                        Avv[a] = Avv[a] + Kvv[nr][nc];
                    }
                }
            }
        }
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Boundary terms of the 3D system (glissade_velo_higher.F90:2848-2898)
// ---------------------------------------------------------------------------
extern "C" {

// dirichlet_boundary_conditions_3d (:9305-9498), loop for loop: vertices j = nhalo..ny-nhalo+1,
// i = nhalo..nx-nhalo+1 that are active, levels k; a u-prescribed node gets b = uvel, a unit
// diagonal, its u-row zeroed and its column moved to the right-hand side of every neighbour
// that is not u- (resp. v-) prescribed; then the same for v.  Masks (nz,nx-1,ny-1) int32 with
// 1 = prescribed; arrays in the caller's layout.
void oracle_dirichlet_3d(int nx, int ny, int nz, int nhalo, const int32_t *active_vertex, const int32_t *umask,
                         const int32_t *vmask, const double *uvel, const double *vvel, double *Auu, double *Auv,
                         double *Avu, double *Avv, double *bu, double *bv) {
    const long NX = nx - 1;
    auto V = [&](int k, int i, int j) { return (long)(k - 1) + (long)nz * ((i - 1) + NX * (j - 1)); };
    auto A = [&](int m, int k, int i, int j) { return (long)(m - 1) + 27L * V(k, i, j); };
    auto M = [](int iA, int jA, int kA) { return 1 + (iA + 1) + 3 * (jA + 1) + 9 * (kA + 1); };
    for (int j = nhalo; j <= ny - nhalo + 1; ++j)
        for (int i = nhalo; i <= nx - nhalo + 1; ++i) {
            if (!active_vertex[(i - 1) + NX * (j - 1)]) continue;
            for (int k = 1; k <= nz; ++k) {
                for (int pass = 0; pass < 2; ++pass) {
                    const int32_t *mask = pass == 0 ? umask : vmask;
                    if (mask[V(k, i, j)] != 1) continue;
                    const double x = pass == 0 ? uvel[V(k, i, j)] : vvel[V(k, i, j)];
                    (pass == 0 ? bu : bv)[V(k, i, j)] = x;
                    for (int kA = -1; kA <= 1; ++kA)
                        for (int jA = -1; jA <= 1; ++jA)
                            for (int iA = -1; iA <= 1; ++iA) {
                                if (!(k + kA >= 1 && k + kA <= nz && i + iA >= 1 && i + iA <= nx - 1 && j + jA >= 1 &&
                                      j + jA <= ny - 1))
                                    continue;
                                if (iA == 0 && jA == 0 && kA == 0) {
                                    const long a = A(M(0, 0, 0), k, i, j);
                                    if (pass == 0) {
                                        Auu[a] = 1.0;
                                        Auv[a] = 0.0;
                                        Avu[a] = 0.0;
                                    } else {
                                        Auv[a] = 0.0;
                                        Avu[a] = 0.0;
                                        Avv[a] = 1.0;
                                    }
                                    continue;
                                }
                                const long a = A(M(iA, jA, kA), k, i, j);
                                if (pass == 0) {
                                    Auu[a] = 0.0;
                                    Auv[a] = 0.0;
                                } else {
                                    Avu[a] = 0.0;
                                    Avv[a] = 0.0;
                                }
                                const long e = V(k + kA, i + iA, j + jA);
                                const long b = A(M(-iA, -jA, -kA), k + kA, i + iA, j + jA);
                                double *Au = pass == 0 ? Auu : Auv, *Av = pass == 0 ? Avu : Avv;
                                if (umask[e] != 1) {
                                    bu[e] = bu[e] - Au[b] * x;
                                    Au[b] = 0.0;
                                }
                                if (vmask[e] != 1) {
                                    bv[e] = bv[e] - Av[b] * x;
                                    Av[b] = 0.0;
                                }
                            }
                }
            }
        }
}

// basal_sliding_bc_3d (:8815-9129), HO_ASSEMBLE_BETA_LOCAL: staglsrf = glissade_stagger(lsrf)
// (glissade_grid_operators.F90:69-157, all four cells), theta = glissade_slope_angle(staglsrf)
// on the (nx-1, ny-1) grid (:1264-1410: glissade_gradient :309-468 with every edge in the mask,
// glissade_unstagger :226-305 over the inner cells, atan of the gradient's length; the
// parallel_halo that follows returns at once for arrays of that size), then at every active
// vertex the bed diagonal of Auu and Avv (level nz) += dx*dy/vol0 * beta / cos(theta).
// theta (nx-1,ny-1) is returned too.
void oracle_basal_local_3d(int nx, int ny, int nz, double dx, double dy, const int32_t *active_vertex,
                           const double *beta, const double *lsrf, double *Auu, double *Avv, double *theta) {
    const int NX = nx - 1, NY = ny - 1;
    std::vector<double> s((size_t)NX * NY), gx((size_t)(NX - 1) * (NY - 1)), gy(gx.size());
    auto L = [&](int i, int j) { return lsrf[(i - 1) + (long)nx * (j - 1)]; };
    auto S = [&](int i, int j) -> double & { return s[(i - 1) + (size_t)NX * (j - 1)]; };
    for (int j = 1; j <= NY; ++j)
        for (int i = 1; i <= NX; ++i) S(i, j) = (L(i, j + 1) + L(i + 1, j + 1) + L(i, j) + L(i + 1, j)) / 4.0;
    // glissade_gradient on the (NX, NY) grid: all edge masks true for the edges it reads
    for (int j = 1; j <= NY - 1; ++j)
        for (int i = 1; i <= NX - 1; ++i) {
            const double north = (S(i + 1, j + 1) - S(i, j + 1)) / dx, south = (S(i + 1, j) - S(i, j)) / dx;
            gx[(i - 1) + (size_t)(NX - 1) * (j - 1)] = (north + south) / 2.0;
            const double east = (S(i + 1, j + 1) - S(i + 1, j)) / dy, west = (S(i, j + 1) - S(i, j)) / dy;
            gy[(i - 1) + (size_t)(NX - 1) * (j - 1)] = (east + west) / 2.0;
        }
    auto G = [&](const std::vector<double> &g, int i, int j) { return g[(i - 1) + (size_t)(NX - 1) * (j - 1)]; };
    for (int j = 1; j <= NY; ++j)
        for (int i = 1; i <= NX; ++i) {
            double ddx = 0.0, ddy = 0.0;
            if (i >= 2 && i <= NX - 1 && j >= 2 && j <= NY - 1) {
                ddx = (G(gx, i, j) + G(gx, i - 1, j) + G(gx, i, j - 1) + G(gx, i - 1, j - 1)) / 4.0;
                ddy = (G(gy, i, j) + G(gy, i - 1, j) + G(gy, i, j - 1) + G(gy, i - 1, j - 1)) / 4.0;
            }
            const double slope = std::sqrt(ddx * ddx + ddy * ddy);
            theta[(i - 1) + (size_t)NX * (j - 1)] = (slope >= 0.0) ? std::atan(slope) : 0.0;
        }
    for (int j = 1; j <= NY; ++j)
        for (int i = 1; i <= NX; ++i) {
            const long q = (i - 1) + (long)NX * (j - 1);
            if (!active_vertex[q]) continue;
            const long a = 13 + 27L * ((long)(nz - 1) + (long)nz * q);
            Auu[a] = Auu[a] + dx * dy / kVol0 * beta[q] / std::cos(theta[q]);
            Avv[a] = Avv[a] + dx * dy / kVol0 * beta[q] / std::cos(theta[q]);
        }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Boundary terms of the 2D system (glissade_velo_higher.F90:2590-2660)
// ---------------------------------------------------------------------------
extern "C" {

// dirichlet_boundary_conditions_2d (:9133-9301), loop for loop: offsets jA, iA outermost, then
// vertices j = nhalo..ny-nhalo+1, i = nhalo..nx-nhalo+1 that are active; a u-prescribed vertex
// sets its diagonals Auu, Auv and Avu to 1 (the 2D routine's choice), a v-prescribed one Auv
// and Avu to 0 and Avv to 1.  Masks (nx-1,ny-1) int32; A** (nx-1,ny-1,9).
void oracle_dirichlet_2d(int nx, int ny, int nhalo, const int32_t *active_vertex, const int32_t *umask,
                         const int32_t *vmask, const double *uvel, const double *vvel, double *Auu, double *Auv,
                         double *Avu, double *Avv, double *bu, double *bv) {
    const long NX = nx - 1, NQ = NX * (ny - 1);
    auto V = [&](int i, int j) { return (long)(i - 1) + NX * (j - 1); };
    auto A = [&](int i, int j, int m) { return V(i, j) + NQ * (m - 1); };
    auto M = [](int iA, int jA) { return 1 + (iA + 1) + 3 * (jA + 1); };
    for (int jA = -1; jA <= 1; ++jA)
        for (int iA = -1; iA <= 1; ++iA) {
            const int m = M(iA, jA), mm = M(-iA, -jA);
            for (int j = nhalo; j <= ny - nhalo + 1; ++j)
                for (int i = nhalo; i <= nx - nhalo + 1; ++i) {
                    if (!active_vertex[V(i, j)]) continue;
                    for (int pass = 0; pass < 2; ++pass) {
                        if ((pass == 0 ? umask : vmask)[V(i, j)] != 1) continue;
                        const double x = pass == 0 ? uvel[V(i, j)] : vvel[V(i, j)];
                        (pass == 0 ? bu : bv)[V(i, j)] = x;
                        if (!(i + iA >= 1 && i + iA <= nx - 1 && j + jA >= 1 && j + jA <= ny - 1)) continue;
                        if (iA == 0 && jA == 0) {
                            const long d = A(i, j, M(0, 0));
                            if (pass == 0) {
                                Auu[d] = 1.0;
                                Auv[d] = 1.0;
                                Avu[d] = 1.0;
                            } else {
                                Auv[d] = 0.0;
                                Avu[d] = 0.0;
                                Avv[d] = 1.0;
                            }
                            continue;
                        }
                        const long a = A(i, j, m);
                        if (pass == 0) {
                            Auu[a] = 0.0;
                            Auv[a] = 0.0;
                        } else {
                            Avu[a] = 0.0;
                            Avv[a] = 0.0;
                        }
                        const long e = V(i + iA, j + jA), b = A(i + iA, j + jA, mm);
                        double *Au = pass == 0 ? Auu : Auv, *Av = pass == 0 ? Avu : Avv;
                        if (umask[e] != 1) {
                            bu[e] = bu[e] - Au[b] * x;
                            Au[b] = 0.0;
                        }
                        if (vmask[e] != 1) {
                            bv[e] = bv[e] - Av[b] * x;
                            Av[b] = 0.0;
                        }
                    }
                }
        }
}

// basal_sliding_bc_2d (:8281-8531), HO_ASSEMBLE_BETA_LOCAL: at every active vertex the
// diagonal of Auu and Avv += (dx*dy/vol0) * beta.
void oracle_basal_local_2d(int nx, int ny, double dx, double dy, const int32_t *active_vertex, const double *beta,
                           double *Auu, double *Avv) {
    const long NQ = (long)(nx - 1) * (ny - 1);
    for (long q = 0; q < NQ; ++q) {
        if (!active_vertex[q]) continue;
        const double increment = (dx * dy / kVol0) * beta[q];
        Auu[q + 4 * NQ] = Auu[q + 4 * NQ] + increment;
        Avv[q + 4 * NQ] = Avv[q + 4 * NQ] + increment;
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// basal_sliding_bc_3d / _2d, standard finite-element form (whichassemble_beta = 0)
// ---------------------------------------------------------------------------
extern "C" {

// basal_sliding_bc_3d (:8876-8960) and basal_sliding_bc_2d (:8337-8410), standard form: every
// active cell j = nhalo+1..ny-nhalo+1, i = nhalo+1..nx-nhalo+1, 4 Gauss points; beta at the
// point from the 4 vertex values; the area factor is get_area_scale_factor_curved_2d
// (:6736-6827, the lower surface staggered over all four cells as z) in 3D and the flat
// Jacobian of get_basis_function_derivatives_2d in 2D; each point's 4x4 matrix
// beta_qp*w*detJ/vol0*phi_r*phi_c is added to Auu and Avv (3D: the bed level nz) at once.
// is3d: blocks (27,nz,nx-1,ny-1), else (nx-1,ny-1,9).  Returns 1 for a singular 2D Jacobian.
int oracle_basal_standard(int is3d, int nx, int ny, int nz, int nhalo, const int32_t *active_cell,
                          const double *xVertex, const double *yVertex, const double *beta, const double *lsrf,
                          double *Auu, double *Avv) {
    const long NX = nx - 1, NQ = NX * (ny - 1);
    const RefElement2 &R = ref2();
    std::vector<double> stag((size_t)NQ, 0.0);
    if (is3d)
        for (int j = 1; j <= ny - 1; ++j)
            for (int i = 1; i <= nx - 1; ++i) {
                auto L = [&](int ii, int jj) { return lsrf[(ii - 1) + (long)nx * (jj - 1)]; };
                stag[(i - 1) + NX * (j - 1)] = (L(i, j + 1) + L(i + 1, j + 1) + L(i, j) + L(i + 1, j)) / 4.0;
            }
    for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
        for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
            if (!active_cell[(i - 1) + (long)nx * (j - 1)]) continue;
            double x[4], y[4], z[4], b[4];
            for (int n = 0; n < 4; ++n) {
                const long q = (long)(i + kIsh3[n] - 1) + NX * (j + kJsh3[n] - 1);
                x[n] = xVertex[q];
                y[n] = yVertex[q];
                z[n] = stag[q];
                b[n] = beta[q];
            }
            for (int p = 0; p < 4; ++p) {
                double detJ;
                if (is3d) {  // get_area_scale_factor_curved_2d
                    double J11 = 0.0, J12 = 0.0, J13 = 0.0, J21 = 0.0, J22 = 0.0, J23 = 0.0;
                    for (int n = 0; n < 4; ++n) {
                        J11 = J11 + R.dxr[p][n] * x[n];
                        J12 = J12 + R.dxr[p][n] * y[n];
                        J13 = J13 + R.dxr[p][n] * z[n];
                        J21 = J21 + R.dyr[p][n] * x[n];
                        J22 = J22 + R.dyr[p][n] * y[n];
                        J23 = J23 + R.dyr[p][n] * z[n];
                    }
                    const double t1 = (J11 * J22 - J12 * J21);
                    const double t2 = -(J11 * J23 - J13 * J21);
                    const double t3 = (J12 * J23 - J13 * J22);
                    detJ = std::sqrt(t1 * t1 + t2 * t2 + t3 * t3);
                } else {
                    double dx[4], dy[4];
                    if (!basis_derivs_2d(x, y, R.dxr[p], R.dyr[p], dx, dy, &detJ)) return 1;
                }
                double beta_qp = 0.0;
                for (int n = 0; n < 4; ++n) beta_qp = beta_qp + R.phi[p][n] * b[n];
                double K[4][4] = {};
                for (int nc = 0; nc < 4; ++nc)
                    for (int nr = 0; nr < 4; ++nr)
                        K[nr][nc] = K[nr][nc] + beta_qp * 1.0 * detJ / kVol0 * R.phi[p][nr] * R.phi[p][nc];
                for (int nr = 0; nr < 4; ++nr) {
                    const long q = (long)(i + kIsh3[nr] - 1) + NX * (j + kJsh3[nr] - 1);
                    for (int nc = 0; nc < 4; ++nc) {
                        const int m = (kIsh3[nc] - kIsh3[nr] + 1) + 3 * (kJsh3[nc] - kJsh3[nr] + 1);  // kA = 0
                        const size_t a = is3d ? (size_t)(m + 9) + 27 * ((size_t)(nz - 1) + (size_t)nz * q)
                                              : (size_t)q + (size_t)NQ * m;
                        Auu[a] = Auu[a] + K[nr][nc];
                        Avv[a] = Avv[a] + K[nr][nc];
                    }
                }
            }
        }
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// assemble_stiffness_matrix_2d, DIVA branch
// ---------------------------------------------------------------------------
namespace {

// compute_effective_viscosity_diva (:7730-7997), the iterative (non-cubic) form, for one
// quadrature point of a 4-node cell: efvs(1:nz-1) enters holding the previous iteration's
// values (0: not yet set) and leaves holding the new ones.
void efvs_diva(int whichefvs, double efvs_constant, double effstrain_min, double n_glen, int nz,
               const double *stagsigma, const double *phi, const double *dx, const double *dy, const double *u,
               const double *v, const double *bx, const double *by, double dsfx, double dsfy, const double *flwafact,
               double *efvs) {
    const double p_effstr = (1.0 - n_glen) / n_glen;
    if (whichefvs == kEfvsConstant) {
        for (int k = 0; k < nz - 1; ++k) efvs[k] = efvs_constant;
        return;
    }
    if (whichefvs == kEfvsFlowfact) {
        const double effstrain = kVeloScale / kLenScale * kScyr;
        for (int k = 0; k < nz - 1; ++k) efvs[k] = flwafact[k] * std::pow(effstrain, p_effstr);
        return;
    }
    double du_dx = 0.0, du_dy = 0.0, dv_dx = 0.0, dv_dy = 0.0, taux = 0.0, tauy = 0.0;
    for (int n = 0; n < 4; ++n) {
        du_dx = du_dx + dx[n] * u[n];
        du_dy = du_dy + dy[n] * u[n];
        dv_dx = dv_dx + dx[n] * v[n];
        dv_dy = dv_dy + dy[n] * v[n];
        taux = taux + phi[n] * bx[n];
        tauy = tauy + phi[n] * by[n];
    }
    for (int k = 0; k < nz - 1; ++k) {
        if (efvs[k] == 0.0) efvs[k] = flwafact[k] * std::pow(effstrain_min, p_effstr);
        const double du_dz = taux * stagsigma[k] / (efvs[k] * dsfx);
        const double dv_dz = tauy * stagsigma[k] / (efvs[k] * dsfy);
        const double sq = effstrain_min * effstrain_min + du_dx * du_dx + dv_dy * dv_dy + du_dx * dv_dy +
                          0.25 * ((dv_dx + du_dy) * (dv_dx + du_dy)) + 0.25 * (du_dz * du_dz) * dsfx +
                          0.25 * (dv_dz * dv_dz) * dsfy;
        efvs[k] = flwafact[k] * std::pow(sq, p_effstr / 2.0);
    }
}

}  // namespace

extern "C" {

// assemble_stiffness_matrix_2d (:4961-5378) with whichapprox = HO_APPROX_DIVA: per active cell and
// Gauss point, the layer viscosities of compute_effective_viscosity_diva from the stored ones
// (efvs_qp_3d (nz-1,4,nx,ny), updated in place), their sigma-weighted average, the element
// matrix of the Blatter-Pattyn form with dphi_dz = 0 and h*efvs; efvs(k,i,j) the mean over the
// points per layer; compute_integrals_diva (:5649-5775) into omega_k (nz,nx,ny) and omega
// (nx,ny) of active cells.  Returns 0, 1 (singular Jacobian) or 2 (nhalo < 2).
int oracle_assemble_stiffness_2d_diva(int nx, int ny, int nz, int nhalo, const double *sigma, const double *stagsigma,
                                      const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                      const double *uvel, const double *vvel, const double *stagthck,
                                      const double *thck, const double *btractx, const double *btracty,
                                      const double *dsfx, const double *dsfy, const double *flwafact, int whichefvs,
                                      double efvs_constant, double effstrain_min, double n_glen, double *efvs_qp_3d,
                                      double *efvs, double *omega_k, double *omega, double *Auu, double *Auv,
                                      double *Avu, double *Avv) {
    if (nhalo < 2) return 2;
    const long NX = nx - 1, NY = ny - 1, NQ = NX * NY;
    const RefElement2 &R = ref2();
    std::memset(efvs, 0, sizeof(double) * (size_t)(nz - 1) * nx * ny);
    for (double *A : {Auu, Auv, Avu, Avv}) std::memset(A, 0, sizeof(double) * 9 * (size_t)NQ);
    for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
        for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
            const long cidx = (i - 1) + (long)nx * (j - 1);
            if (!active_cell[cidx]) continue;
            double Kuu[4][4] = {}, Kuv[4][4] = {}, Kvu[4][4] = {}, Kvv[4][4] = {};
            double x[4], y[4], u[4], v[4], h[4], bx[4], by[4];
            for (int n = 0; n < 4; ++n) {
                const long q = (long)(i + kIsh3[n] - 1) + NX * (j + kJsh3[n] - 1);
                x[n] = xVertex[q];
                y[n] = yVertex[q];
                u[n] = uvel[q];
                v[n] = vvel[q];
                h[n] = stagthck[q];
                bx[n] = btractx[q];
                by[n] = btracty[q];
            }
            double *eq = efvs_qp_3d + (size_t)(nz - 1) * 4 * cidx;  // (nz-1, 4) of this cell
            const double *ff = flwafact + (size_t)(nz - 1) * cidx;
            for (int p = 0; p < 4; ++p) {
                double dx[4], dy[4], dz[4] = {0.0, 0.0, 0.0, 0.0}, detJ;
                if (!basis_derivs_2d(x, y, R.dxr[p], R.dyr[p], dx, dy, &detJ)) return 1;
                efvs_diva(whichefvs, efvs_constant, effstrain_min, n_glen, nz, stagsigma, R.phi[p], dx, dy, u, v, bx, by,
                          dsfx[cidx], dsfy[cidx], ff, eq + (size_t)(nz - 1) * p);
                double vavg = 0.0;
                for (int k = 0; k < nz - 1; ++k) vavg = vavg + eq[(size_t)(nz - 1) * p + k] * (sigma[k + 1] - sigma[k]);
                double h_qp = 0.0;
                for (int n = 0; n < 4; ++n) h_qp = h_qp + R.phi[p][n] * h[n];
                const double f = h_qp * vavg * 1.0 * detJ / kVol0;
                for (int nc = 0; nc < 4; ++nc)
                    for (int nr = 0; nr < 4; ++nr) {
                        Kuu[nr][nc] = Kuu[nr][nc] + f * (4.0 * dx[nr] * dx[nc] + dy[nr] * dy[nc] + dz[nr] * dz[nc]);
                        Kuv[nr][nc] = Kuv[nr][nc] + f * (2.0 * dx[nr] * dy[nc] + dy[nr] * dx[nc]);
                        Kvu[nr][nc] = Kvu[nr][nc] + f * (2.0 * dy[nr] * dx[nc] + dx[nr] * dy[nc]);
                        Kvv[nr][nc] = Kvv[nr][nc] + f * (4.0 * dy[nr] * dy[nc] + dx[nr] * dx[nc] + dz[nr] * dz[nc]);
                    }
            }
            // compute_integrals_diva: omega_kp per point from the bed up, then means over the points
            std::vector<double> okp((size_t)nz * 4);
            for (int p = 0; p < 4; ++p) {
                okp[(size_t)(nz - 1) * 4 + p] = 0.0;
                for (int k = nz - 2; k >= 0; --k) {
                    const double depth = 0.5 * (sigma[k] + sigma[k + 1]);
                    const double dzk = (sigma[k + 1] - sigma[k]) * thck[cidx];
                    okp[(size_t)k * 4 + p] = okp[(size_t)(k + 1) * 4 + p] + depth / eq[(size_t)(nz - 1) * p + k] * dzk;
                }
            }
            double *ok = omega_k + (size_t)nz * cidx;
            for (int k = 0; k < nz; ++k) {
                double sum = 0.0;
                for (int p = 0; p < 4; ++p) sum = sum + okp[(size_t)k * 4 + p];
                ok[k] = sum / 4;
            }
            double om = 0.0;
            for (int k = 0; k < nz - 1; ++k) om = om + 0.5 * (ok[k] + ok[k + 1]) * (sigma[k + 1] - sigma[k]);
            omega[cidx] = om;
            for (int k = 0; k < nz - 1; ++k) {
                double &e = efvs[k + (long)(nz - 1) * cidx];
                e = 0.0;
            }
            for (int p = 0; p < 4; ++p)
                for (int k = 0; k < nz - 1; ++k) {
                    double &e = efvs[k + (long)(nz - 1) * cidx];
                    e = e + eq[(size_t)(nz - 1) * p + k];
                }
            for (int k = 0; k < nz - 1; ++k) efvs[k + (long)(nz - 1) * cidx] /= 4;
            for (int nr = 0; nr < 4; ++nr) {
                const long q = (long)(i + kIsh3[nr] - 1) + NX * (j + kJsh3[nr] - 1);
                for (int nc = 0; nc < 4; ++nc) {
                    const int m = (kIsh3[nc] - kIsh3[nr] + 1) + 3 * (kJsh3[nc] - kJsh3[nr] + 1);
                    const size_t a = (size_t)q + (size_t)NQ * m;
                    Auu[a] = Auu[a] + Kuu[nr][nc];
                    Auv[a] = Auv[a] + Kuv[nr][nc];
                    Avu[a] = Avu[a] + Kvu[nr][nc];
                    Avv[a] = Avv[a] + Kvv[nr][nc];
                }
            }
        }
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// basal_sliding_bc_2d_diva (:8535-8811), the DIVA basal term with slope correction
// ---------------------------------------------------------------------------
extern "C" {

// Local form (whichassemble_beta = 1): theta_x = atan(|dz/dx|), theta_y = atan(|dz/dy|) of the
// staggered lower surface (glissade_slope_angle's theta_slope_x/_y: the gradient and unstagger
// of oracle_basal_local_3d), then at active vertices Auu(0,0) += (dx*dy/vol0)*beta_eff_x/cos(theta_x)
// and Avv(0,0) += (dx*dy/vol0)*beta_eff_y/cos(theta_y).  Standard form (0): per active cell the
// curved area factor of the staggered lower surface and 4-point quadrature, beta_eff_x into Auu
// and beta_eff_y into Avv.  Blocks (nx-1,ny-1,9).
void oracle_basal_diva(int nx, int ny, int nhalo, double dx, double dy, const int32_t *active_cell,
                       const int32_t *active_vertex, const double *bex, const double *bey, const double *lsrf,
                       const double *xVertex, const double *yVertex, int whichassemble_beta, double *Auu, double *Avv) {
    const long NX = nx - 1, NY = ny - 1, NQ = NX * NY;
    auto L = [&](long i, long j) { return lsrf[(i - 1) + (long)nx * (j - 1)]; };
    std::vector<double> s((size_t)NQ);
    for (long j = 1; j <= NY; ++j)
        for (long i = 1; i <= NX; ++i) s[(i - 1) + NX * (j - 1)] = (L(i, j + 1) + L(i + 1, j + 1) + L(i, j) + L(i + 1, j)) / 4.0;
    auto S = [&](long i, long j) { return s[(i - 1) + NX * (j - 1)]; };
    if (whichassemble_beta == 1) {
        std::vector<double> gx((size_t)(NX - 1) * (NY - 1)), gy(gx.size());
        for (long j = 1; j <= NY - 1; ++j)
            for (long i = 1; i <= NX - 1; ++i) {
                const double north = (S(i + 1, j + 1) - S(i, j + 1)) / dx, south = (S(i + 1, j) - S(i, j)) / dx;
                gx[(i - 1) + (NX - 1) * (j - 1)] = (north + south) / 2.0;
                const double east = (S(i + 1, j + 1) - S(i + 1, j)) / dy, west = (S(i, j + 1) - S(i, j)) / dy;
                gy[(i - 1) + (NX - 1) * (j - 1)] = (east + west) / 2.0;
            }
        auto G = [&](const std::vector<double> &g, long i, long j) { return g[(i - 1) + (NX - 1) * (j - 1)]; };
        for (long j = 1; j <= NY; ++j)
            for (long i = 1; i <= NX; ++i) {
                const long q = (i - 1) + NX * (j - 1);
                if (!active_vertex[q]) continue;
                double ddx = 0.0, ddy = 0.0;
                if (i >= 2 && i <= NX - 1 && j >= 2 && j <= NY - 1) {
                    ddx = (G(gx, i, j) + G(gx, i - 1, j) + G(gx, i, j - 1) + G(gx, i - 1, j - 1)) / 4.0;
                    ddy = (G(gy, i, j) + G(gy, i - 1, j) + G(gy, i, j - 1) + G(gy, i - 1, j - 1)) / 4.0;
                }
                const double tx = std::atan(std::fabs(ddx)), ty = std::atan(std::fabs(ddy));
                Auu[q + 4 * NQ] = Auu[q + 4 * NQ] + (dx * dy / kVol0) * bex[q] / std::cos(tx);
                Avv[q + 4 * NQ] = Avv[q + 4 * NQ] + (dx * dy / kVol0) * bey[q] / std::cos(ty);
            }
        return;
    }
    const RefElement2 &R = ref2();
    for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
        for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
            if (!active_cell[(i - 1) + (long)nx * (j - 1)]) continue;
            double x[4], y[4], z[4], bx[4], by[4];
            for (int n = 0; n < 4; ++n) {
                const long q = (long)(i + kIsh3[n] - 1) + NX * (j + kJsh3[n] - 1);
                x[n] = xVertex[q];
                y[n] = yVertex[q];
                z[n] = s[q];
                bx[n] = bex[q];
                by[n] = bey[q];
            }
            for (int p = 0; p < 4; ++p) {
                double J11 = 0.0, J12 = 0.0, J13 = 0.0, J21 = 0.0, J22 = 0.0, J23 = 0.0;
                for (int n = 0; n < 4; ++n) {
                    J11 = J11 + R.dxr[p][n] * x[n];
                    J12 = J12 + R.dxr[p][n] * y[n];
                    J13 = J13 + R.dxr[p][n] * z[n];
                    J21 = J21 + R.dyr[p][n] * x[n];
                    J22 = J22 + R.dyr[p][n] * y[n];
                    J23 = J23 + R.dyr[p][n] * z[n];
                }
                const double t1 = (J11 * J22 - J12 * J21), t2 = -(J11 * J23 - J13 * J21), t3 = (J12 * J23 - J13 * J22);
                const double detJ = std::sqrt(t1 * t1 + t2 * t2 + t3 * t3);
                double bqx = 0.0, bqy = 0.0;
                for (int n = 0; n < 4; ++n) {
                    bqx = bqx + R.phi[p][n] * bx[n];
                    bqy = bqy + R.phi[p][n] * by[n];
                }
                double Ku[4][4] = {}, Kv[4][4] = {};
                for (int nc = 0; nc < 4; ++nc)
                    for (int nr = 0; nr < 4; ++nr) {
                        Ku[nr][nc] = Ku[nr][nc] + bqx * 1.0 * detJ / kVol0 * R.phi[p][nr] * R.phi[p][nc];
                        Kv[nr][nc] = Kv[nr][nc] + bqy * 1.0 * detJ / kVol0 * R.phi[p][nr] * R.phi[p][nc];
                    }
                for (int nr = 0; nr < 4; ++nr) {
                    const long q = (long)(i + kIsh3[nr] - 1) + NX * (j + kJsh3[nr] - 1);
                    for (int nc = 0; nc < 4; ++nc) {
                        const int m = (kIsh3[nc] - kIsh3[nr] + 1) + 3 * (kJsh3[nc] - kJsh3[nr] + 1);
                        Auu[q + NQ * m] = Auu[q + NQ * m] + Ku[nr][nc];
                        Avv[q + NQ * m] = Avv[q + NQ * m] + Kv[nr][nc];
                    }
                }
            }
        }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// assemble_stiffness_matrix_2d, L1L2 branch (compute_effective_viscosity_L1L2 :7474-7726)
// ---------------------------------------------------------------------------
namespace {
constexpr double kRhoi = 910.0, kGrav = 9.81;  // glimmer_physcon.F90:67, :69

// compute_effective_viscosity_L1L2 at one quadrature point of a 4-node cell: per layer the
// cubic for tau_parallel, then efvs = 1/(2A) (n = 1) or 1/(2A(tau_par^2 + tau_perp^2)) (n = 3).
// Fortran's a**3 is (a*a)*a, x**(1/3) is pow.  Returns false for another n_glen (GM_FATAL).
bool efvs_l1l2(int whichefvs, double efvs_constant, double effstrain_min, double n_glen, int nz, const double *sigma,
               const double *phi, const double *dx, const double *dy, const double *u, const double *v,
               const double *h, const double *dsdx, const double *dsdy, const double *flwa, const double *flwafact,
               double *efvs) {
    const double p_effstr = (1.0 - n_glen) / n_glen;
    if (whichefvs == kEfvsConstant) {
        for (int k = 0; k < nz - 1; ++k) efvs[k] = efvs_constant;
        return true;
    }
    if (whichefvs == kEfvsFlowfact) {
        const double effstrain = kVeloScale / kLenScale * kScyr;
        for (int k = 0; k < nz - 1; ++k) efvs[k] = flwafact[k] * std::pow(effstrain, p_effstr);
        return true;
    }
    double du_dx = 0.0, du_dy = 0.0, dv_dx = 0.0, dv_dy = 0.0, ds_dx = 0.0, ds_dy = 0.0, thck = 0.0;
    for (int n = 0; n < 4; ++n) {
        du_dx = du_dx + dx[n] * u[n];
        du_dy = du_dy + dy[n] * u[n];
        dv_dx = dv_dx + dx[n] * v[n];
        dv_dy = dv_dy + dy[n] * v[n];
        ds_dx = ds_dx + phi[n] * dsdx[n];
        ds_dy = ds_dy + phi[n] * dsdy[n];
        thck = thck + phi[n] * h[n];
    }
    const double sq = effstrain_min * effstrain_min + du_dx * du_dx + dv_dy * dv_dy + du_dx * dv_dy +
                      0.25 * ((dv_dx + du_dy) * (dv_dx + du_dy));
    const double effstrain = std::sqrt(sq);
    for (int k = 0; k < nz - 1; ++k) {
        const double depth = thck * sigma[k + 1];
        const double grads = std::sqrt(ds_dx * ds_dx + ds_dy * ds_dy);
        const double tau_perp = kRhoi * kGrav * depth * grads;
        const double a = tau_perp * tau_perp;
        const double b = -effstrain / flwa[k];
        const double a3 = (a * a) * a;
        const double c = std::sqrt(b * b / 4.0 + a3 / 27.0);
        const double rootA = std::pow(-b / 2.0 + c, 1.0 / 3.0);
        double rootB;
        if (a3 / 27.0 > 1.0e-6 * (b * b / 4.0)) rootB = -std::pow(b / 2.0 + c, 1.0 / 3.0);
        else rootB = -a / (3.0 * std::pow(std::fabs(b), 1.0 / 3.0));
        const double tau_parallel = rootA + rootB;
        if (std::fabs(n_glen - 1.0) < 1.0e-10) efvs[k] = 1.0 / (2.0 * flwa[k]);
        else if (std::fabs(n_glen - 3.0) < 1.0e-10)
            efvs[k] = 1.0 / (2.0 * flwa[k] * (tau_parallel * tau_parallel + tau_perp * tau_perp));
        else return false;
    }
    return true;
}
}  // namespace

extern "C" {

// assemble_stiffness_matrix_2d (:4961-5378) with whichapprox = HO_APPROX_L1L2: per Gauss point the
// layer viscosities of compute_effective_viscosity_L1L2 (surface gradient dusrf_dx/_dy at the
// vertices, flwa per layer), their sigma-weighted average, the Blatter-Pattyn element matrix with
// dphi_dz = 0 and h*efvs; efvs(k,i,j) the mean over the points.  Returns 0, 1 (singular Jacobian),
// 2 (nhalo < 2) or 3 (n_glen neither 1 nor 3, the reference's GM_FATAL).
int oracle_assemble_stiffness_2d_l1l2(int nx, int ny, int nz, int nhalo, const double *sigma,
                                      const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                      const double *uvel, const double *vvel, const double *stagthck,
                                      const double *dusrf_dx, const double *dusrf_dy, const double *flwa,
                                      const double *flwafact, int whichefvs, double efvs_constant,
                                      double effstrain_min, double n_glen, double *efvs, double *Auu, double *Auv,
                                      double *Avu, double *Avv) {
    if (nhalo < 2) return 2;
    const long NX = nx - 1, NY = ny - 1, NQ = NX * NY;
    const RefElement2 &R = ref2();
    std::memset(efvs, 0, sizeof(double) * (size_t)(nz - 1) * nx * ny);
    for (double *A : {Auu, Auv, Avu, Avv}) std::memset(A, 0, sizeof(double) * 9 * (size_t)NQ);
    std::vector<double> eq((size_t)(nz - 1) * 4);
    for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
        for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
            const long cidx = (i - 1) + (long)nx * (j - 1);
            if (!active_cell[cidx]) continue;
            double Kuu[4][4] = {}, Kuv[4][4] = {}, Kvu[4][4] = {}, Kvv[4][4] = {};
            double x[4], y[4], u[4], v[4], h[4], sx[4], sy[4];
            for (int n = 0; n < 4; ++n) {
                const long q = (long)(i + kIsh3[n] - 1) + NX * (j + kJsh3[n] - 1);
                x[n] = xVertex[q];
                y[n] = yVertex[q];
                u[n] = uvel[q];
                v[n] = vvel[q];
                h[n] = stagthck[q];
                sx[n] = dusrf_dx[q];
                sy[n] = dusrf_dy[q];
            }
            const double *fl = flwa + (size_t)(nz - 1) * cidx, *ff = flwafact + (size_t)(nz - 1) * cidx;
            for (int p = 0; p < 4; ++p) {
                double dx[4], dy[4], dz[4] = {0.0, 0.0, 0.0, 0.0}, detJ;
                if (!basis_derivs_2d(x, y, R.dxr[p], R.dyr[p], dx, dy, &detJ)) return 1;
                double *e = eq.data() + (size_t)(nz - 1) * p;
                if (!efvs_l1l2(whichefvs, efvs_constant, effstrain_min, n_glen, nz, sigma, R.phi[p], dx, dy, u, v, h,
                               sx, sy, fl, ff, e))
                    return 3;
                double vavg = 0.0;
                for (int k = 0; k < nz - 1; ++k) vavg = vavg + e[k] * (sigma[k + 1] - sigma[k]);
                double h_qp = 0.0;
                for (int n = 0; n < 4; ++n) h_qp = h_qp + R.phi[p][n] * h[n];
                const double f = h_qp * vavg * 1.0 * detJ / kVol0;
                for (int nc = 0; nc < 4; ++nc)
                    for (int nr = 0; nr < 4; ++nr) {
                        Kuu[nr][nc] = Kuu[nr][nc] + f * (4.0 * dx[nr] * dx[nc] + dy[nr] * dy[nc] + dz[nr] * dz[nc]);
                        Kuv[nr][nc] = Kuv[nr][nc] + f * (2.0 * dx[nr] * dy[nc] + dy[nr] * dx[nc]);
                        Kvu[nr][nc] = Kvu[nr][nc] + f * (2.0 * dy[nr] * dx[nc] + dx[nr] * dy[nc]);
                        Kvv[nr][nc] = Kvv[nr][nc] + f * (4.0 * dy[nr] * dy[nc] + dx[nr] * dx[nc] + dz[nr] * dz[nc]);
                    }
            }
            for (int k = 0; k < nz - 1; ++k) {
                double s = 0.0;
                for (int p = 0; p < 4; ++p) s = s + eq[(size_t)(nz - 1) * p + k];
                efvs[k + (long)(nz - 1) * cidx] = s / 4;
            }
            for (int nr = 0; nr < 4; ++nr) {
                const long q = (long)(i + kIsh3[nr] - 1) + NX * (j + kJsh3[nr] - 1);
                for (int nc = 0; nc < 4; ++nc) {
                    const int m = (kIsh3[nc] - kIsh3[nr] + 1) + 3 * (kJsh3[nc] - kJsh3[nr] + 1);
                    const size_t a = (size_t)q + (size_t)NQ * m;
                    Auu[a] = Auu[a] + Kuu[nr][nc];
                    Auv[a] = Auv[a] + Kuv[nr][nc];
                    Avu[a] = Avu[a] + Kvu[nr][nc];
                    Avv[a] = Avv[a] + Kvv[nr][nc];
                }
            }
        }
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// load_vector_gravity (:4228-4449)
// ---------------------------------------------------------------------------
extern "C" {

// Local form (whichassemble_taud = 1): at every active vertex and level k,
// load -= rhoi*grav*dx*dy*dz/vol0 * dusrf_dx with dz = stagthck*(stagwbndsigma(k) -
// stagwbndsigma(k-1)).  Standard form (0): per active cell and element, 8-point quadrature of
// rhoi*grav*w*detJ/vol0 * (ds/dx at the point) * phi_n into each node.  loadu/loadv
// (nz,nx-1,ny-1) are added to (the reference's caller zeroes them); stagwbndsigma (0:nz).
// Returns 0, 1 (singular Jacobian) or 2 (nhalo < 2).
int oracle_load_vector_gravity(int nx, int ny, int nz, int nhalo, const double *sigma, const double *stagwbndsigma,
                               double dx, double dy, const int32_t *active_cell, const int32_t *active_vertex,
                               const double *xVertex, const double *yVertex, const double *stagusrf,
                               const double *stagthck, const double *dusrf_dx, const double *dusrf_dy,
                               int whichassemble_taud, double *loadu, double *loadv) {
    const long NX = nx - 1;
    auto V = [&](int k, int i, int j) { return (long)(k - 1) + (long)nz * ((i - 1) + NX * (j - 1)); };
    if (whichassemble_taud == 1) {
        for (int j = 1; j <= ny - 1; ++j)
            for (int i = 1; i <= nx - 1; ++i) {
                const long q = (i - 1) + NX * (j - 1);
                if (!active_vertex[q]) continue;
                for (int k = 1; k <= nz; ++k) {
                    const double dz = stagthck[q] * (stagwbndsigma[k] - stagwbndsigma[k - 1]);
                    loadu[V(k, i, j)] = loadu[V(k, i, j)] - kRhoi * kGrav * dx * dy * dz / kVol0 * dusrf_dx[q];
                    loadv[V(k, i, j)] = loadv[V(k, i, j)] - kRhoi * kGrav * dx * dy * dz / kVol0 * dusrf_dy[q];
                }
            }
        return 0;
    }
    if (nhalo < 2) return 2;
    const RefElement &R = ref();
    double phi[8][8];  // phi_3d(n,p) at the Gauss points, :354-361
    {
        const double r = 1.0 / std::sqrt(3.0);
        const double xq[8] = {-r, r, r, -r, -r, r, r, -r}, yq[8] = {-r, -r, r, r, -r, -r, r, r},
                     zq[8] = {-r, -r, -r, -r, r, r, r, r};
        for (int p = 0; p < 8; ++p) {
            const double x = xq[p], y = yq[p], z = zq[p];
            phi[p][0] = (1.0 - x) * (1.0 - y) * (1.0 - z) / 8.0;
            phi[p][1] = (1.0 + x) * (1.0 - y) * (1.0 - z) / 8.0;
            phi[p][2] = (1.0 + x) * (1.0 + y) * (1.0 - z) / 8.0;
            phi[p][3] = (1.0 - x) * (1.0 + y) * (1.0 - z) / 8.0;
            phi[p][4] = (1.0 - x) * (1.0 - y) * (1.0 + z) / 8.0;
            phi[p][5] = (1.0 + x) * (1.0 - y) * (1.0 + z) / 8.0;
            phi[p][6] = (1.0 + x) * (1.0 + y) * (1.0 + z) / 8.0;
            phi[p][7] = (1.0 - x) * (1.0 + y) * (1.0 + z) / 8.0;
        }
    }
    for (int j = nhalo + 1; j <= ny - nhalo + 1; ++j)
        for (int i = nhalo + 1; i <= nx - nhalo + 1; ++i) {
            if (!active_cell[(i - 1) + (long)nx * (j - 1)]) continue;
            for (int k = 1; k <= nz - 1; ++k) {
                double x[8], y[8], z[8], sx[8], sy[8];
                for (int n = 0; n < 8; ++n) {
                    const long q = (long)(i + kIsh7[n] - 1) + NX * (j + kJsh7[n] - 1);
                    x[n] = xVertex[q];
                    y[n] = yVertex[q];
                    z[n] = stagusrf[q] - sigma[k + kKsh7[n] - 1] * stagthck[q];
                    sx[n] = dusrf_dx[q];
                    sy[n] = dusrf_dy[q];
                }
                for (int p = 0; p < 8; ++p) {
                    double ddx[8], ddy[8], ddz[8], detJ;
                    if (!basis_derivs_3d(x, y, z, R.dxr[p], R.dyr[p], R.dzr[p], ddx, ddy, ddz, &detJ)) return 1;
                    double sxq = 0.0, syq = 0.0;
                    for (int n = 0; n < 8; ++n) {
                        sxq = sxq + phi[p][n] * sx[n];
                        syq = syq + phi[p][n] * sy[n];
                    }
                    for (int n = 0; n < 8; ++n) {
                        const long e = V(k + kKsh7[n], i + kIsh7[n], j + kJsh7[n]);
                        loadu[e] = loadu[e] - kRhoi * kGrav * R.wqp[p] * detJ / kVol0 * sxq * phi[p][n];
                        loadv[e] = loadv[e] - kRhoi * kGrav * R.wqp[p] * detJ / kVol0 * syq * phi[p][n];
                    }
                }
            }
        }
    return 0;
}

}  // extern "C"
