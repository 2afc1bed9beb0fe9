// assembly.cu -- the Blatter-Pattyn stiffness matrix assembled on the device:
// assemble_stiffness_matrix_3d (libglissade/glissade_velo_higher.F90:5382-5643) with
// get_basis_function_derivatives_3d (:6508-6732), compute_effective_viscosity (:7285-7470),
// compute_element_matrix (:8001-8123) and element_to_global_matrix_3d (:8200-8268).
//
// The reference loops over the elements (active cells j, i, then layers k) and adds each 8x8
// element matrix into the 27-point rows of its 8 nodes.  Here the 3D stiffness is built in two
// kernels per slab of cell rows: k_asm_elements3d evaluates every element's quadrature once
// (the element's 8 Gauss points on 8 threads, shared through shared memory, then its 8 rows on
// 8 threads) into a scratch of element matrices that L2 keeps, and k_asm_gather3d has one
// thread per matrix row (node k, i, j) sum the rows of the (up to) 8 elements that contain its
// node in the reference's element order (j, then i, then k).  Every coefficient thus receives
// the same terms in the same order as in the reference, with no atomics.  The 2D kernels keep
// the gather-and-recompute form (4-point cells, one thread per vertex).
// The arithmetic is the reference's operation for operation (the library is built without FMA
// contraction); only pow (the flow law's (effstrain^2)^((1-n)/2n), and the flow-factor option's
// power, which the host evaluates once) is CUDA's rather than the host C library's.

namespace cismgpu {

constexpr double kAsmVol0 = 1.0e9;   // vol0, glissade_velo_higher.F90:1254
constexpr int kAsmBlock = 128;

// The reference element (glissade_velo_higher.F90:314-392): weights and the derivatives of the
// 8 trilinear basis functions at the 8 Gauss points, filled by the host.
struct AsmRef {
    double wqp[8];
    double dxr[8][8], dyr[8][8], dzr[8][8];  // [p][n]
    double phi[8][8];                        // phi_3d(n,p) at [p][n] (:354-361)
};
__constant__ AsmRef c_asm_ref;

// node n of an element relative to node 7 (ishift(7,n), jshift(7,n), kshift(7,n), :455-478)
__constant__ int c_ish7[8] = {-1, 0, 0, -1, -1, 0, 0, -1};
__constant__ int c_jsh7[8] = {-1, -1, 0, 0, -1, -1, 0, 0};
__constant__ int c_ksh7[8] = {1, 1, 1, 1, 0, 0, 0, 0};

struct AsmArgs {
    int nx, ny, nz, nhalo;
    int whichapprox, whichefvs;  // 0 SIA, 1 SSA, else BP; 0 constant, 1 flow factor, 2 nonlinear
    double efvs_constant, effstrain_min, p_half;  // p_half = (1 - n)/n / 2
    double flowfact_pow;                          // (velo_scale/len_scale*scyr)^((1-n)/n), host pow
    const double *sigma;                          // (nz)
    const int32_t *active_cell;                   // (nx, ny)
    const double *xv, *yv, *usrf, *thck;          // (nx-1, ny-1)
    const double *u, *v;                          // (nz, nx-1, ny-1), or level-major planes
    int vel_planes;                               // 1: u, v are level-major planes (k*NQ + q)
    const double *flwafact;                       // (nz-1, nx, ny)
    double *efvs;                                 // (nz-1, nx, ny), zeroed by the host
    int *singular;                                // set when an element's Jacobian is singular
};

// Node n of an element relative to node 7, as constant expressions (the gather below resolves
// its coupling indices at compile time)
__host__ __device__ constexpr int ish7(int n) { return (n == 0 || n == 3 || n == 4 || n == 7) ? -1 : 0; }
__host__ __device__ constexpr int jsh7(int n) { return (n % 4 < 2) ? -1 : 0; }
__host__ __device__ constexpr int ksh7(int n) { return n < 4 ? 1 : 0; }

// Element matrices are built element by element into a scratch of cell-row slabs, then gathered
// node by node.  Scratch layout: K[b][nr][nc][e], b = Kuu, Kuv, Kvu, Kvv, row nr and column nc of
// the 8x8 element matrix, e = (ie-1) + nx*((ke-1) + (nz-1)*(je-je0)) the slab's element index.
constexpr int kAsmEl = 16;                        // elements per block of k_asm_elements3d
constexpr int kAsmElThreads = 8 * kAsmEl;         // one thread per (element, Gauss point / row)
static_assert(kAsmEl == 16, "k_asm_elements3d maps a warp to 2 x 16 elements");
constexpr size_t kAsmScratchBytes = 64ull << 20;  // slab scratch budget (L2 keeps it between the kernels)

// One Gauss point of one element: the basis-function derivatives, the viscosity and the
// quadrature factor efvs * w * detJ / vol0 that every entry of the element matrix takes.
struct AsmPt {
    double dx[8], dy[8], dz[8];
    double f, efvs;
};

// get_basis_function_derivatives_3d (:6508-6732) and compute_effective_viscosity (:7285-7470)
// at Gauss point p of the element with nodes x, y, z, u, v and flow factor ff.  Returns false
// for a singular Jacobian.
__device__ bool asm_point3d(const AsmArgs &a, int p, const double (&x)[8], const double (&y)[8],
                            const double (&z)[8], const double (&u)[8], const double (&v)[8], double ff, AsmPt &o) {
    const double *dxr = c_asm_ref.dxr[p], *dyr = c_asm_ref.dyr[p], *dzr = c_asm_ref.dzr[p];
    double J00 = 0.0, J01 = 0.0, J02 = 0.0, J10 = 0.0, J11 = 0.0, J12 = 0.0, J20 = 0.0, J21 = 0.0, J22 = 0.0;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        J00 = J00 + dxr[n] * x[n];
        J01 = J01 + dxr[n] * y[n];
        J02 = J02 + dxr[n] * z[n];
        J10 = J10 + dyr[n] * x[n];
        J11 = J11 + dyr[n] * y[n];
        J12 = J12 + dyr[n] * z[n];
        J20 = J20 + dzr[n] * x[n];
        J21 = J21 + dzr[n] * y[n];
        J22 = J22 + dzr[n] * z[n];
    }
    const double c00 = J11 * J22 - J12 * J21, c01 = -(J10 * J22 - J12 * J20), c02 = J10 * J21 - J11 * J20;
    const double c10 = -(J01 * J22 - J02 * J21), c11 = J00 * J22 - J02 * J20, c12 = -(J00 * J21 - J01 * J20);
    const double c20 = J01 * J12 - J02 * J11, c21 = -(J00 * J12 - J02 * J10), c22 = J00 * J11 - J01 * J10;
    const double detJ = J00 * c00 + J01 * c01 + J02 * c02;
    if (!(fabs(detJ) > 0.0)) return false;
    // Jinv(row,col) = cofactor(col,row) / detJ
    const double i00 = c00 / detJ, i01 = c10 / detJ, i02 = c20 / detJ;
    const double i10 = c01 / detJ, i11 = c11 / detJ, i12 = c21 / detJ;
    const double i20 = c02 / detJ, i21 = c12 / detJ, i22 = c22 / detJ;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        o.dx[n] = i00 * dxr[n] + i01 * dyr[n] + i02 * dzr[n];
        o.dy[n] = i10 * dxr[n] + i11 * dyr[n] + i12 * dzr[n];
        o.dz[n] = i20 * dxr[n] + i21 * dyr[n] + i22 * dzr[n];
    }
    double efvs;
    if (a.whichefvs == 0) {
        efvs = a.efvs_constant;
    } else if (a.whichefvs == 1) {
        efvs = ff * a.flowfact_pow;
    } else {
        double du_dx = 0.0, du_dy = 0.0, du_dz = 0.0, dv_dx = 0.0, dv_dy = 0.0, dv_dz = 0.0, sq;
        const double em2 = a.effstrain_min * a.effstrain_min;
        if (a.whichapprox == 0) {
#pragma unroll
            for (int n = 0; n < 8; ++n) {
                du_dz = du_dz + o.dz[n] * u[n];
                dv_dz = dv_dz + o.dz[n] * v[n];
            }
            sq = em2 + 0.25 * (du_dz * du_dz + dv_dz * dv_dz);
        } else {
#pragma unroll
            for (int n = 0; n < 8; ++n) {
                du_dx = du_dx + o.dx[n] * u[n];
                du_dy = du_dy + o.dy[n] * u[n];
                if (a.whichapprox != 1) du_dz = du_dz + o.dz[n] * u[n];
                dv_dx = dv_dx + o.dx[n] * v[n];
                dv_dy = dv_dy + o.dy[n] * v[n];
                if (a.whichapprox != 1) dv_dz = dv_dz + o.dz[n] * v[n];
            }
            const double sh = dv_dx + du_dy;
            sq = em2 + (du_dx * du_dx + dv_dy * dv_dy + du_dx * dv_dy + 0.25 * (sh * sh));
            if (a.whichapprox != 1) sq = sq + 0.25 * (du_dz * du_dz + dv_dz * dv_dz);
        }
        efvs = ff * pow(sq, a.p_half);
    }
    o.efvs = efvs;
    o.f = efvs * c_asm_ref.wqp[p] * detJ / kAsmVol0;
    return true;
}

// The element matrices of the cell rows je0 .. je0+nrows-1 (1-based), every layer: the
// reference's element loop body (:5502-5581), each element's quadrature evaluated once.  A block
// holds kAsmEl elements.  Phase 1, thread (element, p): the element's nodes and Gauss point p
// into shared memory.  Phase 2, 8 threads an element: the four 8x8 blocks,
// compute_element_matrix (:8001-8123) over the points in order, into the scratch K.  An element
// outside the reference's cell loop (nhalo+1..n-nhalo+1) or inactive writes nothing (the gather
// never reads it).  Its first thread writes the element's mean viscosity (:5575-5581) when its
// own node (ie-1, je-1, ke-1) is a vertex with je-1 in [jown0, jown1).
__global__ void __launch_bounds__(kAsmElThreads) k_asm_elements3d(AsmArgs a, int je0, int nrows, int jown0,
                                                                  int jown1, double *__restrict__ K, long long ks) {
    __shared__ AsmPt sp[8][kAsmEl];
    const int nzl1 = a.nz - 1;
    const long long nel = (long long)a.nx * nzl1 * nrows;
    const long long NX = a.nx - 1;
    const int tid = threadIdx.x, el = tid % kAsmEl, sub = tid / kAsmEl;
    const long long e = (long long)blockIdx.x * kAsmEl + el;
    int ie = 0, je = 0, ke = 0;
    bool valid = false;
    if (e < nel) {
        ie = (int)(e % a.nx) + 1;
        const long long r = e / a.nx;
        ke = (int)(r % nzl1) + 1;
        je = je0 + (int)(r / nzl1);
        valid = ie >= a.nhalo + 1 && ie <= a.nx - a.nhalo + 1 && je >= a.nhalo + 1 && je <= a.ny - a.nhalo + 1 &&
                a.active_cell[(ie - 1) + (long long)a.nx * (je - 1)] != 0;
    }
    if (valid) {  // phase 1: Gauss point p = sub
        double x[8], y[8], z[8], u[8], v[8];
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            const int iN = ie + ish7(n), jN = je + jsh7(n), kN = ke + ksh7(n);
            const long long q = (long long)(iN - 1) + NX * (jN - 1);
            x[n] = a.xv[q];
            y[n] = a.yv[q];
            z[n] = a.usrf[q] - a.sigma[kN - 1] * a.thck[q];
            const long long ev = a.vel_planes ? (long long)(kN - 1) * NX * (a.ny - 1) + q : (long long)(kN - 1) + a.nz * q;
            u[n] = a.u[ev];
            v[n] = a.v[ev];
        }
        const double ff = a.flwafact[(ke - 1) + (long long)nzl1 * ((ie - 1) + (long long)a.nx * (je - 1))];
        if (!asm_point3d(a, sub, x, y, z, u, v, ff, sp[sub][el])) atomicExch(a.singular, 1);
    }
    __syncthreads();
    if (!valid) return;
    // phase 2.  The blocks' entries are products the reference forms in an order that makes
    // Kuu and Kvv symmetric and Kvu the transpose of Kuv bit for bit ((4 a) b and (4 b) a, (2 a) b
    // and (2 b) a round the same exact product; a b = b a).  Warp w (r = w) takes rows r and
    // 7 - r of the upper triangle (columns >= the row, 9 entries, written with their mirrors)
    // of Kuu in its first half-warp and of Kvv in its second, and each thread one row of Kuv
    // (urow = 2 w + half, written with its transpose in Kvu): 17 entries a thread instead of
    // 32, warp-uniform, each summed over the points in order, as compute_element_matrix does.
    // Kvv's entries are Kuu's with dx and dy exchanged: 4 dy dy + dx dx (+ dz dz).
    const int r = tid / 32, comp = (tid / kAsmEl) % 2, r2 = 7 - r, urow = 2 * r + comp;
    double U[8], Sa[8], Sb[8];  // Kuv row urow; rows r (columns >= r) and 7 - r (columns >= 7 - r)
#pragma unroll
    for (int nc = 0; nc < 8; ++nc) U[nc] = Sa[nc] = Sb[nc] = 0.0;
    for (int p = 0; p < 8; ++p) {
        const AsmPt &P = sp[p][el];
        const double f = P.f;
        const double *p1 = comp == 0 ? P.dx : P.dy, *p2 = comp == 0 ? P.dy : P.dx;
        const double a1 = p1[r], a2 = p2[r], az = P.dz[r];
        const double b1 = p1[r2], b2 = p2[r2], bz = P.dz[r2];
        const double ux = P.dx[urow], uy = P.dy[urow];
#pragma unroll
        for (int nc = 0; nc < 8; ++nc) {
            const double cx = P.dx[nc], cy = P.dy[nc], cz = P.dz[nc];
            const double c1 = comp == 0 ? cx : cy, c2 = comp == 0 ? cy : cx;
            if (a.whichapprox != 0) U[nc] = U[nc] + f * (2.0 * ux * cy + uy * cx);
            if (a.whichapprox == 0) {
                if (nc >= r) Sa[nc] = Sa[nc] + f * (az * cz);
                if (nc >= r2) Sb[nc] = Sb[nc] + f * (bz * cz);
            } else if (a.whichapprox == 1) {
                if (nc >= r) Sa[nc] = Sa[nc] + f * (4.0 * a1 * c1 + a2 * c2);
                if (nc >= r2) Sb[nc] = Sb[nc] + f * (4.0 * b1 * c1 + b2 * c2);
            } else {
                if (nc >= r) Sa[nc] = Sa[nc] + f * (4.0 * a1 * c1 + a2 * c2 + az * cz);
                if (nc >= r2) Sb[nc] = Sb[nc] + f * (4.0 * b1 * c1 + b2 * c2 + bz * cz);
            }
        }
    }
    const int bs = comp == 0 ? 0 : 3;  // Kuu or Kvv
#pragma unroll
    for (int nc = 0; nc < 8; ++nc) {
        if (nc >= r) {
            K[(long long)((bs * 8 + r) * 8 + nc) * ks + e] = Sa[nc];
            if (nc != r) K[(long long)((bs * 8 + nc) * 8 + r) * ks + e] = Sa[nc];
        }
        if (nc >= r2) {
            K[(long long)((bs * 8 + r2) * 8 + nc) * ks + e] = Sb[nc];
            if (nc != r2) K[(long long)((bs * 8 + nc) * 8 + r2) * ks + e] = Sb[nc];
        }
        K[(long long)((1 * 8 + urow) * 8 + nc) * ks + e] = U[nc];  // Kuv(urow, nc)
        K[(long long)((2 * 8 + nc) * 8 + urow) * ks + e] = U[nc];  // Kvu(nc, urow)
    }
    if (sub == 0 && ie - 1 < NX && je - 1 < a.ny - 1 && je - 1 >= jown0 && je - 1 < jown1) {
        double esum = 0.0;
        for (int p = 0; p < 8; ++p) esum = esum + sp[p][el].efvs;
        a.efvs[(ke - 1) + (long long)nzl1 * ((ie - 1) + (long long)a.nx * (je - 1))] = esum / 8;
    }
}

// Element slot s = 4 dj + 2 di + dk of a node (the element at cell (i+1+di, j+1+dj), layer k+dk,
// 1-based node (i, j, k)): the node's row in that element (shifts (-di, -dj, 1-dk) from node 7),
// and the element column that lands on the node's coupling m, or -1.
__host__ __device__ constexpr int asm_slot_row(int s) {
    return ((s % 2) == 0 ? 0 : 4) + ((s / 4) == 0 ? (((s / 2) % 2) == 0 ? 2 : 3) : (((s / 2) % 2) == 0 ? 1 : 0));
}
__host__ __device__ constexpr int asm_col_coupling(int nr, int nc) {
    return (ish7(nc) - ish7(nr) + 1) + 3 * (jsh7(nc) - jsh7(nr) + 1) + 9 * (ksh7(nc) - ksh7(nr) + 1);
}
__host__ __device__ constexpr int asm_slot_col(int s, int m) {
    return asm_col_coupling(asm_slot_row(s), 0) == m ? 0
         : asm_col_coupling(asm_slot_row(s), 1) == m ? 1
         : asm_col_coupling(asm_slot_row(s), 2) == m ? 2
         : asm_col_coupling(asm_slot_row(s), 3) == m ? 3
         : asm_col_coupling(asm_slot_row(s), 4) == m ? 4
         : asm_col_coupling(asm_slot_row(s), 5) == m ? 5
         : asm_col_coupling(asm_slot_row(s), 6) == m ? 6
         : asm_col_coupling(asm_slot_row(s), 7) == m ? 7 : -1;
}

// element_to_global_matrix_3d (:8200-8268) as a gather: one thread per node (k0, i0, j0),
// 0-based, of the vertex rows j0 in [ja, jb), and block b = blockIdx.y, over the (up to) 8
// elements that contain the node in the reference's element order (j, then i, then k), each
// valid when its cell is one the reference loops over, is active, and its layer exists.  The coefficient for coupling m of
// block b sums, in that order, the column of the element's row for the node that lands on m
// (slot, row and column are compile-time constants: one running sum at a time).
// Every coefficient of every node in the rows is written, zero where no element contributes
// (the reference zeroes A first).  je0: the scratch slab's first cell row.
__global__ void __launch_bounds__(kAsmBlock) k_asm_gather3d(AsmArgs a, SymIdx L, int ja, int jb, int je0,
                                                            const double *__restrict__ K, long long ks,
                                                            double *Auu, double *Auv, double *Avu, double *Avv) {
    const long long NX = a.nx - 1;
    const long long nrow = (long long)(jb - ja) * NX;
    const long long t = (long long)blockIdx.x * kAsmBlock + threadIdx.x;
    if (t >= (long long)a.nz * nrow) return;
    const int k0 = (int)(t / nrow);
    const long long rem = t - (long long)k0 * nrow;
    const int j0 = ja + (int)(rem / NX), i0 = (int)(rem % NX);
    const long long q = (long long)j0 * NX + i0;
    const int iR = i0 + 1, jR = j0 + 1, kR = k0 + 1;
    const int nzl1 = a.nz - 1;
    long long es[8];
    bool ok[8];
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int dj = s / 4, di = (s / 2) % 2, dk = s % 2;
        const int je = jR + dj, ie = iR + di, ke = kR - 1 + dk;
        ok[s] = ke >= 1 && ke <= nzl1 && ie >= a.nhalo + 1 && ie <= a.nx - a.nhalo + 1 && je >= a.nhalo + 1 &&
                je <= a.ny - a.nhalo + 1 && a.active_cell[(ie - 1) + (long long)a.nx * (je - 1)] != 0;
        es[s] = (long long)(ie - 1) + (long long)a.nx * ((ke - 1) + (long long)nzl1 * (je - je0));
    }
    const int b = blockIdx.y;  // the block: Kuu, Kuv, Kvu, Kvv
    const double *Kb = K + (long long)(b * 64) * ks;
    double *Bb = b == 0 ? Auu : b == 1 ? Auv : b == 2 ? Avu : Avv;
#pragma unroll
    for (int m = 0; m < 27; ++m) {
        double acc = 0.0;
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            const int nc = asm_slot_col(s, m);
            if (nc >= 0 && ok[s]) acc = acc + Kb[(long long)(asm_slot_row(s) * 8 + nc) * ks + es[s]];
        }
        Bb[L.at(m, k0, q)] = acc;
    }
}

// ---------------------------------------------------------------------------
// assemble_stiffness_matrix_2d (glissade_velo_higher.F90:4961-5378), SSA branch: 4-node
// quadrilaterals, 4 Gauss points (:528-570), get_basis_function_derivatives_2d (:6319-6504),
// the SSA viscosity at the layer-averaged flow factor, h at the point, and
// element_to_global_matrix_2d (:8127-8196).  One thread per vertex, gathering the (up to) 4
// cells around it in the reference's cell order (j, then i).
// ---------------------------------------------------------------------------
struct AsmRef2 {
    double phi[4][4], dxr[4][4], dyr[4][4];  // [p][n]
};
__constant__ AsmRef2 c_asm_ref2;
__constant__ int c_ish3[4] = {-1, 0, 0, -1};  // ishift(3,n), jshift(3,n), n = 1..4
__constant__ int c_jsh3[4] = {-1, -1, 0, 0};

// glissade_vertical_average (glissade_grid_operators.F90:1882-1946, no mask) of flwafact
// (nz-1, nx, ny) into ff2 (nx, ny): sum over k of flwafact(k) * (sigma(k+1) - sigma(k)).
__global__ void __launch_bounds__(kBlock) k_asm_vertavg(int ncell, int nz, const double *__restrict__ sigma,
                                                       const double *__restrict__ ff, double *__restrict__ ff2) {
    const int c = blockIdx.x * kBlock + threadIdx.x;
    if (c >= ncell) return;
    double f = 0.0;
    for (int k = 0; k < nz - 1; ++k) f = f + ff[k + (long long)(nz - 1) * c] * (sigma[k + 1] - sigma[k]);
    ff2[c] = f;
}

// Row nr of cell (ie, je)'s element matrix into acc[b][m]; the cell's own thread writes its
// efvs for every layer (the mean over the 4 points, :5348-5354).
__device__ bool asm_cell_row(const AsmArgs &a, const double *ff2, int ie, int je, int nr, bool own,
                             double acc[4][9]) {
    const long long NX = a.nx - 1;
    double x[4], y[4], u[4], v[4], h[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        const long long q = (long long)(ie + c_ish3[n] - 1) + NX * (je + c_jsh3[n] - 1);
        x[n] = a.xv[q];
        y[n] = a.yv[q];
        u[n] = a.u[q];
        v[n] = a.v[q];
        h[n] = a.thck[q];
    }
    const double ffc = ff2[(ie - 1) + (long long)a.nx * (je - 1)];
    double Kuu[4], Kuv[4], Kvu[4], Kvv[4];
#pragma unroll
    for (int nc = 0; nc < 4; ++nc) Kuu[nc] = Kuv[nc] = Kvu[nc] = Kvv[nc] = 0.0;
    double esum = 0.0;
    for (int p = 0; p < 4; ++p) {
        const double *dxr = c_asm_ref2.dxr[p], *dyr = c_asm_ref2.dyr[p];
        double J00 = 0.0, J01 = 0.0, J10 = 0.0, J11 = 0.0;
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            J00 = J00 + dxr[n] * x[n];
            J01 = J01 + dxr[n] * y[n];
            J10 = J10 + dyr[n] * x[n];
            J11 = J11 + dyr[n] * y[n];
        }
        const double detJ = J00 * J11 - J01 * J10;
        if (!(fabs(detJ) > 0.0)) return false;
        const double i00 = J11 / detJ, i01 = -J01 / detJ, i10 = -J10 / detJ, i11 = J00 / detJ;
        double dx[4], dy[4];
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            dx[n] = 0.0 + i00 * dxr[n] + i01 * dyr[n];
            dy[n] = 0.0 + i10 * dxr[n] + i11 * dyr[n];
        }
        double efvs;
        if (a.whichefvs == 0) {
            efvs = a.efvs_constant;
        } else if (a.whichefvs == 1) {
            efvs = ffc * a.flowfact_pow;
        } else {
            double du_dx = 0.0, du_dy = 0.0, dv_dx = 0.0, dv_dy = 0.0;
#pragma unroll
            for (int n = 0; n < 4; ++n) {
                du_dx = du_dx + dx[n] * u[n];
                du_dy = du_dy + dy[n] * u[n];
                dv_dx = dv_dx + dx[n] * v[n];
                dv_dy = dv_dy + dy[n] * v[n];
            }
            const double sh = dv_dx + du_dy;
            const double sq = a.effstrain_min * a.effstrain_min +
                              (du_dx * du_dx + dv_dy * dv_dy + du_dx * dv_dy + 0.25 * (sh * sh));
            efvs = ffc * pow(sq, a.p_half);
        }
        esum = esum + efvs;
        double h_qp = 0.0;
#pragma unroll
        for (int n = 0; n < 4; ++n) h_qp = h_qp + c_asm_ref2.phi[p][n] * h[n];
        const double f = h_qp * efvs * 1.0 * detJ / kAsmVol0;
#pragma unroll
        for (int nc = 0; nc < 4; ++nc) {
            Kuu[nc] = Kuu[nc] + f * (4.0 * dx[nr] * dx[nc] + dy[nr] * dy[nc]);
            Kuv[nc] = Kuv[nc] + f * (2.0 * dx[nr] * dy[nc] + dy[nr] * dx[nc]);
            Kvu[nc] = Kvu[nc] + f * (2.0 * dy[nr] * dx[nc] + dx[nr] * dy[nc]);
            Kvv[nc] = Kvv[nc] + f * (4.0 * dy[nr] * dy[nc] + dx[nr] * dx[nc]);
        }
    }
    if (own) {
        const double e = esum / 4;
        for (int k = 0; k < a.nz - 1; ++k) a.efvs[k + (long long)(a.nz - 1) * ((ie - 1) + (long long)a.nx * (je - 1))] = e;
    }
#pragma unroll
    for (int nc = 0; nc < 4; ++nc) {
        const int m = (c_ish3[nc] - c_ish3[nr] + 1) + 3 * (c_jsh3[nc] - c_jsh3[nr] + 1);
        acc[0][m] = acc[0][m] + Kuu[nc];
        acc[1][m] = acc[1][m] + Kuv[nc];
        acc[2][m] = acc[2][m] + Kvu[nc];
        acc[3][m] = acc[3][m] + Kvv[nc];
    }
    return true;
}

__global__ void __launch_bounds__(kAsmBlock) k_assemble2d(AsmArgs a, const double *__restrict__ ff2, SymIdx L,
                                                          double *Auu, double *Auv, double *Avu, double *Avv) {
    const long long NX = a.nx - 1, NQ = NX * (a.ny - 1);
    const long long q = (long long)blockIdx.x * kAsmBlock + threadIdx.x;
    if (q >= NQ) return;
    const int j0 = (int)(q / NX), i0 = (int)(q - (long long)j0 * NX);
    const int iR = i0 + 1, jR = j0 + 1;
    double acc[4][9];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int c = 0; c < 9; ++c) acc[b][c] = 0.0;
    for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
            const int je = jR + dj, ie = iR + di;
            if (ie < a.nhalo + 1 || ie > a.nx - a.nhalo + 1 || je < a.nhalo + 1 || je > a.ny - a.nhalo + 1) continue;
            if (!a.active_cell[(ie - 1) + (long long)a.nx * (je - 1)]) continue;
            // node index within the cell: shifts (iR-ie, jR-je) = (-di, -dj)
            const int nr = dj == 0 ? (di == 0 ? 2 : 3) : (di == 0 ? 1 : 0);
            if (!asm_cell_row(a, ff2, ie, je, nr, dj == 0 && di == 0, acc)) atomicExch(a.singular, 1);
        }
    double *B[4] = {Auu, Auv, Avu, Avv};
#pragma unroll
    for (int b = 0; b < 4; ++b)
        for (int c = 0; c < 9; ++c) B[b][L.at(c, 0, q)] = acc[b][c];
}

// ---------------------------------------------------------------------------
// Boundary terms of the 3D system (glissade_velo_higher.F90:2848-2898)
// ---------------------------------------------------------------------------
// Vector element (k, q) of a (nz, nx-1, ny-1) field: the caller's layout or level-major planes.
// The Dirichlet pass takes one for b, one for the masks and one for the velocity, which on a
// handle come from the device planes and the host respectively.
struct VecIdx {
    long long NQ;
    int nz;
    int planes;
    __device__ __forceinline__ long long at(int k, long long q) const {
        return planes ? (long long)k * NQ + q : (long long)k + (long long)nz * q;
    }
};

// dirichlet_boundary_conditions_3d (:9305-9498), one thread per node P.  The reference loops
// over the prescribed nodes R (vertices j = nhalo..ny-nhalo+1, i = nhalo..nx-nhalo+1, active;
// levels k; u then v) and (a) rewrites R's own row and b(R), (b) moves R's column into the
// right-hand side of each neighbour P not prescribed in that component and zeroes the
// coupling.  Every write of (a) and (b) lands in row P or b(P) of a single P, and (b) reads
// only row P's couplings to R, which nothing else writes: so each P applies, in the
// reference's order of R (j, then i, then k; u before v), the moves from its prescribed
// neighbours, and then, when P itself is a visited prescribed node, its own row.  b enters
// holding the load vector.
__global__ void __launch_bounds__(kBlock) k_dirichlet3d(int nx, int ny, int nz, int nhalo, SymIdx L, VecIdx Wb,
                                                        VecIdx Wm, VecIdx Wx,
                                                        const int32_t *__restrict__ active_vertex,
                                                        const int32_t *__restrict__ umask,
                                                        const int32_t *__restrict__ vmask,
                                                        const double *__restrict__ uvel,
                                                        const double *__restrict__ vvel, double *Auu, double *Auv,
                                                        double *Avu, double *Avv, double *bu, double *bv) {
    const long long NX = nx - 1, NQ = NX * (ny - 1);
    const long long t = (long long)blockIdx.x * kBlock + threadIdx.x;
    if (t >= (long long)nz * NQ) return;
    const int k = (int)(t / NQ);
    const long long q = t - (long long)k * NQ;
    const int j = (int)(q / NX), i = (int)(q - (long long)j * NX);  // 0-based
    // a node's own pass runs when its vertex is in the loop range (1-based nhalo..n-nhalo+1)
    // and active
    auto visited = [&](int ii, int jj) {
        return ii >= nhalo - 1 && ii <= nx - nhalo && jj >= nhalo - 1 && jj <= ny - nhalo &&
               active_vertex[(long long)jj * NX + ii] != 0;
    };
    const long long bP = Wb.at(k, q), mP = Wm.at(k, q), xP = Wx.at(k, q);
    const bool ufree = umask[mP] != 1, vfree = vmask[mP] != 1;
    double b_u = bu[bP], b_v = bv[bP];
    for (int ej = -1; ej <= 1; ++ej)
        for (int ei = -1; ei <= 1; ++ei)
            for (int ek = -1; ek <= 1; ++ek) {
                if (ei == 0 && ej == 0 && ek == 0) continue;
                const int kR = k + ek, iR = i + ei, jR = j + ej;
                if (kR < 0 || kR >= nz || iR < 0 || iR >= NX || jR < 0 || jR >= ny - 1) continue;
                if (!visited(iR, jR)) continue;
                const long long qR = (long long)jR * NX + iR, mR = Wm.at(kR, qR), xR = Wx.at(kR, qR);
                const int c = (ei + 1) + 3 * (ej + 1) + 9 * (ek + 1);  // row P's coupling to R
                const long long a = L.at(c, k, q);
                if (umask[mR] == 1) {
                    const double x = uvel[xR];
                    if (ufree) {
                        b_u = b_u - Auu[a] * x;
                        Auu[a] = 0.0;
                    }
                    if (vfree) {
                        b_v = b_v - Avu[a] * x;
                        Avu[a] = 0.0;
                    }
                }
                if (vmask[mR] == 1) {
                    const double x = vvel[xR];
                    if (ufree) {
                        b_u = b_u - Auv[a] * x;
                        Auv[a] = 0.0;
                    }
                    if (vfree) {
                        b_v = b_v - Avv[a] * x;
                        Avv[a] = 0.0;
                    }
                }
            }
    if (visited(i, j)) {
        for (int pass = 0; pass < 2; ++pass) {
            if ((pass == 0 ? umask : vmask)[mP] != 1) continue;
            if (pass == 0) b_u = uvel[xP];
            else b_v = vvel[xP];
            for (int c = 0; c < 27; ++c) {
                const int ei = c % 3 - 1, ej = (c / 3) % 3 - 1, ek = c / 9 - 1;
                if (k + ek < 0 || k + ek >= nz || i + ei < 0 || i + ei >= NX || j + ej < 0 || j + ej >= ny - 1)
                    continue;
                const long long a = L.at(c, k, q);
                if (c == 13) {
                    if (pass == 0) {
                        Auu[a] = 1.0;
                        Auv[a] = 0.0;
                        Avu[a] = 0.0;
                    } else {
                        Auv[a] = 0.0;
                        Avu[a] = 0.0;
                        Avv[a] = 1.0;
                    }
                } else if (pass == 0) {
                    Auu[a] = 0.0;
                    Auv[a] = 0.0;
                } else {
                    Avu[a] = 0.0;
                    Avv[a] = 0.0;
                }
            }
        }
    }
    bu[bP] = b_u;
    bv[bP] = b_v;
}

// basal_sliding_bc_3d with HO_ASSEMBLE_BETA_LOCAL (:8840-8875), one thread per vertex: the
// slope angle of the staggered lower surface (glissade_stagger of lsrf over all four cells,
// glissade_gradient with every edge, glissade_unstagger over the inner vertices, atan), each
// intermediate recomputed from its inputs in the reference's operation order, then at an
// active vertex the bed diagonal (level nz) of Auu and Avv += dx*dy/vol0 * beta / cos(theta).
__global__ void __launch_bounds__(kBlock) k_basal_local3d(int nx, int ny, int nz, double dx, double dy, SymIdx L,
                                                          const int32_t *__restrict__ active_vertex,
                                                          const double *__restrict__ beta,
                                                          const double *__restrict__ lsrf, double *Auu,
                                                          double *Avv) {
    const int NX = nx - 1, NY = ny - 1;
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    if (q >= (long long)NX * NY) return;
    if (!active_vertex[q]) return;
    const int j = (int)(q / NX) + 1, i = (int)(q - (long long)(j - 1) * NX) + 1;  // 1-based
    auto Lf = [&](int ii, int jj) { return lsrf[(ii - 1) + (long long)nx * (jj - 1)]; };
    auto S = [&](int ii, int jj) { return (Lf(ii, jj + 1) + Lf(ii + 1, jj + 1) + Lf(ii, jj) + Lf(ii + 1, jj)) / 4.0; };
    double ddx = 0.0, ddy = 0.0;
    if (i >= 2 && i <= NX - 1 && j >= 2 && j <= NY - 1) {
        double gx[4], gy[4];  // at (i,j), (i-1,j), (i,j-1), (i-1,j-1)
        const int oi[4] = {0, -1, 0, -1}, oj[4] = {0, 0, -1, -1};
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            const int a = i + oi[n], b = j + oj[n];
            const double s00 = S(a, b), s10 = S(a + 1, b), s01 = S(a, b + 1), s11 = S(a + 1, b + 1);
            const double north = (s11 - s01) / dx, south = (s10 - s00) / dx;
            gx[n] = (north + south) / 2.0;
            const double east = (s11 - s10) / dy, west = (s01 - s00) / dy;
            gy[n] = (east + west) / 2.0;
        }
        ddx = (gx[0] + gx[1] + gx[2] + gx[3]) / 4.0;
        ddy = (gy[0] + gy[1] + gy[2] + gy[3]) / 4.0;
    }
    const double slope = sqrt(ddx * ddx + ddy * ddy);
    const double theta = (slope >= 0.0) ? atan(slope) : 0.0;
    const double add = dx * dy / kAsmVol0 * beta[q] / cos(theta);
    const long long a = L.at(13, nz - 1, q);
    Auu[a] = Auu[a] + add;
    Avv[a] = Avv[a] + add;
}

// ---------------------------------------------------------------------------
// Boundary terms of the 2D system (glissade_velo_higher.F90:2590-2660)
// ---------------------------------------------------------------------------
// dirichlet_boundary_conditions_2d (:9133-9301), one thread per vertex P.  The reference loops
// over the offsets (jA, iA) outermost and the prescribed vertices R inside, so the moves into
// b(P) come in the order of the offset P - R (jA, then iA), u before v for each R; every write
// lands in row P or b(P) as in 3D.  A u-prescribed vertex's own diagonals Auu, Auv, Avu become
// 1 (the 2D routine's rule), a v-prescribed one's Auv, Avu 0 and Avv 1, u before v.  Masks,
// velocities and b in the (nx-1, ny-1) layout; blocks in layout L (NC = 9).
__global__ void __launch_bounds__(kBlock) k_dirichlet2d(int nx, int ny, int nhalo, SymIdx L,
                                                        const int32_t *__restrict__ active_vertex,
                                                        const int32_t *__restrict__ umask,
                                                        const int32_t *__restrict__ vmask,
                                                        const double *__restrict__ uvel,
                                                        const double *__restrict__ vvel, double *Auu, double *Auv,
                                                        double *Avu, double *Avv, double *bu, double *bv) {
    const long long NX = nx - 1, NQ = NX * (ny - 1);
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    if (q >= NQ) return;
    const int j = (int)(q / NX), i = (int)(q - (long long)j * NX);  // 0-based
    auto visited = [&](int ii, int jj) {
        return ii >= nhalo - 1 && ii <= nx - nhalo && jj >= nhalo - 1 && jj <= ny - nhalo &&
               active_vertex[(long long)jj * NX + ii] != 0;
    };
    const bool ufree = umask[q] != 1, vfree = vmask[q] != 1;
    double b_u = bu[q], b_v = bv[q];
    for (int jA = -1; jA <= 1; ++jA)
        for (int iA = -1; iA <= 1; ++iA) {
            if (iA == 0 && jA == 0) continue;
            const int iR = i - iA, jR = j - jA;  // P = R + (iA, jA)
            if (iR < 0 || iR >= NX || jR < 0 || jR >= ny - 1) continue;
            if (!visited(iR, jR)) continue;
            const long long qR = (long long)jR * NX + iR;
            const int c = (-iA + 1) + 3 * (-jA + 1);  // row P's coupling to R
            const long long a = L.at(c, 0, q);
            if (umask[qR] == 1) {
                const double x = uvel[qR];
                if (ufree) {
                    b_u = b_u - Auu[a] * x;
                    Auu[a] = 0.0;
                }
                if (vfree) {
                    b_v = b_v - Avu[a] * x;
                    Avu[a] = 0.0;
                }
            }
            if (vmask[qR] == 1) {
                const double x = vvel[qR];
                if (ufree) {
                    b_u = b_u - Auv[a] * x;
                    Auv[a] = 0.0;
                }
                if (vfree) {
                    b_v = b_v - Avv[a] * x;
                    Avv[a] = 0.0;
                }
            }
        }
    if (visited(i, j)) {
        for (int pass = 0; pass < 2; ++pass) {
            if ((pass == 0 ? umask : vmask)[q] != 1) continue;
            if (pass == 0) b_u = uvel[q];
            else b_v = vvel[q];
            for (int c = 0; c < 9; ++c) {
                const int ei = c % 3 - 1, ej = c / 3 - 1;
                if (i + ei < 0 || i + ei >= NX || j + ej < 0 || j + ej >= ny - 1) continue;
                const long long a = L.at(c, 0, q);
                if (c == 4) {
                    if (pass == 0) {
                        Auu[a] = 1.0;
                        Auv[a] = 1.0;
                        Avu[a] = 1.0;
                    } else {
                        Auv[a] = 0.0;
                        Avu[a] = 0.0;
                        Avv[a] = 1.0;
                    }
                } else if (pass == 0) {
                    Auu[a] = 0.0;
                    Auv[a] = 0.0;
                } else {
                    Avu[a] = 0.0;
                    Avv[a] = 0.0;
                }
            }
        }
    }
    bu[q] = b_u;
    bv[q] = b_v;
}

// basal_sliding_bc_2d with HO_ASSEMBLE_BETA_LOCAL (:8325-8336): at every active vertex the
// diagonal of Auu and Avv += (dx*dy/vol0) * beta.
__global__ void __launch_bounds__(kBlock) k_basal_local2d(long long NQ, double dx, double dy, SymIdx L,
                                                          const int32_t *__restrict__ active_vertex,
                                                          const double *__restrict__ beta, double *Auu, double *Avv) {
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    if (q >= NQ || !active_vertex[q]) return;
    const double increment = (dx * dy / kAsmVol0) * beta[q];
    const long long a = L.at(4, 0, q);
    Auu[a] = Auu[a] + increment;
    Avv[a] = Avv[a] + increment;
}

// basal_sliding_bc_3d (:8876-8960) / basal_sliding_bc_2d (:8337-8410), standard finite-element
// form, one thread per vertex: the (up to) 4 active cells around it in the reference's order
// (j, then i), and for each of the cell's 4 Gauss points the vertex's row of
// beta_qp*w*detJ/vol0*phi_r*phi_c added to Auu and Avv, point by point as the reference adds
// them.  3D: the area factor of the lower surface (get_area_scale_factor_curved_2d, :6736-6827,
// lsrf staggered over all four cells) and the bed level nz; 2D: the flat Jacobian, or with
// CURVED the area factor as in 3D (basal_sliding_bc_2d_diva :8650-8700, which also takes a
// separate beta for v, beta_v).
template <bool THREE_D, bool CURVED>
__global__ void __launch_bounds__(kBlock) k_basal_standard(int nx, int ny, int nz, int nhalo, SymIdx L,
                                                           const int32_t *__restrict__ active_cell,
                                                           const double *__restrict__ xv,
                                                           const double *__restrict__ yv,
                                                           const double *__restrict__ beta,
                                                           const double *__restrict__ beta_v,
                                                           const double *__restrict__ lsrf, double *Auu,
                                                           double *Avv, int *singular) {
    const long long NX = nx - 1, NQ = NX * (ny - 1);
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    if (q >= NQ) return;
    const int jR = (int)(q / NX) + 1, iR = (int)(q - (long long)(jR - 1) * NX) + 1;  // 1-based
    auto Lf = [&](int ii, int jj) { return lsrf[(ii - 1) + (long long)nx * (jj - 1)]; };
    const int base = THREE_D ? 9 : 0;  // indxA_3d(iA, jA, 0) = indxA_2d(iA, jA) + 9
    const int lev = THREE_D ? nz - 1 : 0;
    double accU[9], accV[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        accU[c] = Auu[L.at(c + base, lev, q)];
        accV[c] = Avv[L.at(c + base, lev, q)];
    }
    bool any = false;
    for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
            const int je = jR + dj, ie = iR + di;
            if (ie < nhalo + 1 || ie > nx - nhalo + 1 || je < nhalo + 1 || je > ny - nhalo + 1) continue;
            if (!active_cell[(ie - 1) + (long long)nx * (je - 1)]) continue;
            any = true;
            const int nr = dj == 0 ? (di == 0 ? 2 : 3) : (di == 0 ? 1 : 0);
            double x[4], y[4], z[4], b[4], bv[4];
#pragma unroll
            for (int n = 0; n < 4; ++n) {
                const int iN = ie + c_ish3[n], jN = je + c_jsh3[n];
                const long long qn = (long long)(iN - 1) + NX * (jN - 1);
                x[n] = xv[qn];
                y[n] = yv[qn];
                b[n] = beta[qn];
                bv[n] = beta_v[qn];
                z[n] = CURVED ? (Lf(iN, jN + 1) + Lf(iN + 1, jN + 1) + Lf(iN, jN) + Lf(iN + 1, jN)) / 4.0 : 0.0;
            }
            for (int p = 0; p < 4; ++p) {
                const double *dxr = c_asm_ref2.dxr[p], *dyr = c_asm_ref2.dyr[p];
                double detJ;
                if (CURVED) {
                    double J11 = 0.0, J12 = 0.0, J13 = 0.0, J21 = 0.0, J22 = 0.0, J23 = 0.0;
#pragma unroll
                    for (int n = 0; n < 4; ++n) {
                        J11 = J11 + dxr[n] * x[n];
                        J12 = J12 + dxr[n] * y[n];
                        J13 = J13 + dxr[n] * z[n];
                        J21 = J21 + dyr[n] * x[n];
                        J22 = J22 + dyr[n] * y[n];
                        J23 = J23 + dyr[n] * z[n];
                    }
                    const double t1 = (J11 * J22 - J12 * J21);
                    const double t2 = -(J11 * J23 - J13 * J21);
                    const double t3 = (J12 * J23 - J13 * J22);
                    detJ = sqrt(t1 * t1 + t2 * t2 + t3 * t3);
                } else {
                    double J00 = 0.0, J01 = 0.0, J10 = 0.0, J11 = 0.0;
#pragma unroll
                    for (int n = 0; n < 4; ++n) {
                        J00 = J00 + dxr[n] * x[n];
                        J01 = J01 + dxr[n] * y[n];
                        J10 = J10 + dyr[n] * x[n];
                        J11 = J11 + dyr[n] * y[n];
                    }
                    detJ = J00 * J11 - J01 * J10;
                    if (!(fabs(detJ) > 0.0)) {
                        atomicExch(singular, 1);
                        continue;
                    }
                }
                double beta_qp = 0.0, beta_qv = 0.0;
#pragma unroll
                for (int n = 0; n < 4; ++n) {
                    beta_qp = beta_qp + c_asm_ref2.phi[p][n] * b[n];
                    beta_qv = beta_qv + c_asm_ref2.phi[p][n] * bv[n];
                }
#pragma unroll
                for (int nc = 0; nc < 4; ++nc) {
                    const double ku = 0.0 + beta_qp * 1.0 * detJ / kAsmVol0 * c_asm_ref2.phi[p][nr] * c_asm_ref2.phi[p][nc];
                    const double kv = 0.0 + beta_qv * 1.0 * detJ / kAsmVol0 * c_asm_ref2.phi[p][nr] * c_asm_ref2.phi[p][nc];
                    const int m = (c_ish3[nc] - c_ish3[nr] + 1) + 3 * (c_jsh3[nc] - c_jsh3[nr] + 1);
                    accU[m] = accU[m] + ku;
                    accV[m] = accV[m] + kv;
                }
            }
        }
    if (!any) return;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        Auu[L.at(c + base, lev, q)] = accU[c];
        Avv[L.at(c + base, lev, q)] = accV[c];
    }
}

// ---------------------------------------------------------------------------
// assemble_stiffness_matrix_2d, DIVA branch (:5230-5300 with compute_effective_viscosity_diva
// :7730-7997, iterative form, and compute_integrals_diva :5649-5775)
// ---------------------------------------------------------------------------
// The layer viscosities of each cell's Gauss points are state carried between Picard
// iterations (efvs_qp_3d(nz-1, 4, nx, ny)).  Every vertex thread recomputes its cells' new
// viscosities from the previous state; the cell's own thread also writes them, to a second
// buffer, with the cell's efvs, omega_k and omega, so no thread reads what another writes.
struct DivaArgs {
    const double *stagsigma;       // (nz-1)
    const double *thck;            // (nx, ny) cell thickness
    const double *bx, *by;         // (nx-1, ny-1) basal traction
    const double *dsfx, *dsfy;     // (nx, ny) slope factors
    const double *eq_old;          // (nz-1, 4, nx, ny)
    double *eq_new, *omega_k, *omega;
    double init_pow;               // effstrain_min^((1-n)/n), for a state still zero
};

__device__ bool asm_cell_row_diva(const AsmArgs &a, const DivaArgs &d, int ie, int je, int nr, bool own,
                                  double acc[4][9]) {
    const long long NX = a.nx - 1;
    const int nl = a.nz - 1;
    double x[4], y[4], u[4], v[4], h[4], bx[4], by[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        const long long q = (long long)(ie + c_ish3[n] - 1) + NX * (je + c_jsh3[n] - 1);
        x[n] = a.xv[q];
        y[n] = a.yv[q];
        u[n] = a.u[q];
        v[n] = a.v[q];
        h[n] = a.thck[q];
        bx[n] = d.bx[q];
        by[n] = d.by[q];
    }
    const long long cidx = (ie - 1) + (long long)a.nx * (je - 1);
    const double *ff = a.flwafact + (long long)nl * cidx;
    const double *eo = d.eq_old + (long long)nl * 4 * cidx;
    double *en = d.eq_new + (long long)nl * 4 * cidx;
    const double sx = d.dsfx[cidx], sy = d.dsfy[cidx];
    double Kuu[4], Kuv[4], Kvu[4], Kvv[4];
#pragma unroll
    for (int nc = 0; nc < 4; ++nc) Kuu[nc] = Kuv[nc] = Kvu[nc] = Kvv[nc] = 0.0;
    for (int p = 0; p < 4; ++p) {
        const double *dxr = c_asm_ref2.dxr[p], *dyr = c_asm_ref2.dyr[p], *phi = c_asm_ref2.phi[p];
        double J00 = 0.0, J01 = 0.0, J10 = 0.0, J11 = 0.0;
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            J00 = J00 + dxr[n] * x[n];
            J01 = J01 + dxr[n] * y[n];
            J10 = J10 + dyr[n] * x[n];
            J11 = J11 + dyr[n] * y[n];
        }
        const double detJ = J00 * J11 - J01 * J10;
        if (!(fabs(detJ) > 0.0)) return false;
        const double i00 = J11 / detJ, i01 = -J01 / detJ, i10 = -J10 / detJ, i11 = J00 / detJ;
        double dx[4], dy[4];
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            dx[n] = 0.0 + i00 * dxr[n] + i01 * dyr[n];
            dy[n] = 0.0 + i10 * dxr[n] + i11 * dyr[n];
        }
        double du_dx = 0.0, du_dy = 0.0, dv_dx = 0.0, dv_dy = 0.0, taux = 0.0, tauy = 0.0;
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            du_dx = du_dx + dx[n] * u[n];
            du_dy = du_dy + dy[n] * u[n];
            dv_dx = dv_dx + dx[n] * v[n];
            dv_dy = dv_dy + dy[n] * v[n];
            taux = taux + phi[n] * bx[n];
            tauy = tauy + phi[n] * by[n];
        }
        double vavg = 0.0;
        for (int k = 0; k < nl; ++k) {
            double e;
            if (a.whichefvs == 0) {
                e = a.efvs_constant;
            } else if (a.whichefvs == 1) {
                e = ff[k] * a.flowfact_pow;
            } else {
                double eold = eo[(long long)nl * p + k];
                if (eold == 0.0) eold = ff[k] * d.init_pow;
                const double du_dz = taux * d.stagsigma[k] / (eold * sx);
                const double dv_dz = tauy * d.stagsigma[k] / (eold * sy);
                const double sh = dv_dx + du_dy;
                const double sq = a.effstrain_min * a.effstrain_min + du_dx * du_dx + dv_dy * dv_dy + du_dx * dv_dy +
                                  0.25 * (sh * sh) + 0.25 * (du_dz * du_dz) * sx + 0.25 * (dv_dz * dv_dz) * sy;
                e = ff[k] * pow(sq, a.p_half);
            }
            if (own) en[(long long)nl * p + k] = e;
            vavg = vavg + e * (a.sigma[k + 1] - a.sigma[k]);
        }
        double h_qp = 0.0;
#pragma unroll
        for (int n = 0; n < 4; ++n) h_qp = h_qp + phi[n] * h[n];
        const double f = h_qp * vavg * 1.0 * detJ / kAsmVol0;
        const double zero = 0.0 * 0.0;  // dphi_dz(nr)*dphi_dz(nc) of the Blatter-Pattyn form, dphi_dz = 0
#pragma unroll
        for (int nc = 0; nc < 4; ++nc) {
            Kuu[nc] = Kuu[nc] + f * (4.0 * dx[nr] * dx[nc] + dy[nr] * dy[nc] + zero);
            Kuv[nc] = Kuv[nc] + f * (2.0 * dx[nr] * dy[nc] + dy[nr] * dx[nc]);
            Kvu[nc] = Kvu[nc] + f * (2.0 * dy[nr] * dx[nc] + dx[nr] * dy[nc]);
            Kvv[nc] = Kvv[nc] + f * (4.0 * dy[nr] * dy[nc] + dx[nr] * dx[nc] + zero);
        }
    }
    if (own) {
        // efvs(k) = the mean over the points; compute_integrals_diva over the new state
        for (int k = 0; k < nl; ++k) {
            double e = 0.0;
            for (int p = 0; p < 4; ++p) e = e + en[(long long)nl * p + k];
            a.efvs[k + (long long)nl * cidx] = e / 4;
        }
        const double tc = d.thck[cidx];
        double *ok = d.omega_k + (long long)a.nz * cidx;
        double om = 0.0, prev = 0.0;
        // omega_k(k) = (sum over p of the integral from the bed to layer k) / 4, from the bed up
        double okp[4] = {0.0, 0.0, 0.0, 0.0};
        ok[a.nz - 1] = (((0.0 + okp[0]) + okp[1]) + okp[2] + okp[3]) / 4;
        for (int k = nl - 1; k >= 0; --k) {
            const double depth = 0.5 * (a.sigma[k] + a.sigma[k + 1]);
            const double dzk = (a.sigma[k + 1] - a.sigma[k]) * tc;
            double sum = 0.0;
            for (int p = 0; p < 4; ++p) {
                okp[p] = okp[p] + depth / en[(long long)nl * p + k] * dzk;
                sum = sum + okp[p];
            }
            ok[k] = sum / 4;
        }
        for (int k = 0; k < nl; ++k) {
            prev = 0.5 * (ok[k] + ok[k + 1]);
            om = om + prev * (a.sigma[k + 1] - a.sigma[k]);
        }
        d.omega[cidx] = om;
    }
#pragma unroll
    for (int nc = 0; nc < 4; ++nc) {
        const int m = (c_ish3[nc] - c_ish3[nr] + 1) + 3 * (c_jsh3[nc] - c_jsh3[nr] + 1);
        acc[0][m] = acc[0][m] + Kuu[nc];
        acc[1][m] = acc[1][m] + Kuv[nc];
        acc[2][m] = acc[2][m] + Kvu[nc];
        acc[3][m] = acc[3][m] + Kvv[nc];
    }
    return true;
}

__global__ void __launch_bounds__(kAsmBlock) k_assemble2d_diva(AsmArgs a, DivaArgs d, SymIdx L, double *Auu,
                                                               double *Auv, double *Avu, double *Avv) {
    const long long NX = a.nx - 1, NQ = NX * (a.ny - 1);
    const long long q = (long long)blockIdx.x * kAsmBlock + threadIdx.x;
    if (q >= NQ) return;
    const int j0 = (int)(q / NX), i0 = (int)(q - (long long)j0 * NX);
    const int iR = i0 + 1, jR = j0 + 1;
    double acc[4][9];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int c = 0; c < 9; ++c) acc[b][c] = 0.0;
    for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
            const int je = jR + dj, ie = iR + di;
            if (ie < a.nhalo + 1 || ie > a.nx - a.nhalo + 1 || je < a.nhalo + 1 || je > a.ny - a.nhalo + 1) continue;
            if (!a.active_cell[(ie - 1) + (long long)a.nx * (je - 1)]) continue;
            const int nr = dj == 0 ? (di == 0 ? 2 : 3) : (di == 0 ? 1 : 0);
            if (!asm_cell_row_diva(a, d, ie, je, nr, dj == 0 && di == 0, acc)) atomicExch(a.singular, 1);
        }
    double *B[4] = {Auu, Auv, Avu, Avv};
#pragma unroll
    for (int b = 0; b < 4; ++b)
        for (int c = 0; c < 9; ++c) B[b][L.at(c, 0, q)] = acc[b][c];
}

// basal_sliding_bc_2d_diva (:8586-8620), local form, one thread per vertex: glissade_slope_angle's
// theta_x = atan(|dz/dx|), theta_y = atan(|dz/dy|) of the staggered lower surface (the chain of
// k_basal_local3d), then at an active vertex the diagonal of Auu += (dx*dy/vol0)*beta_eff_x /
// cos(theta_x) and of Avv += (dx*dy/vol0)*beta_eff_y / cos(theta_y).
__global__ void __launch_bounds__(kBlock) k_basal_local_diva(int nx, int ny, double dx, double dy, SymIdx L,
                                                             const int32_t *__restrict__ active_vertex,
                                                             const double *__restrict__ bex,
                                                             const double *__restrict__ bey,
                                                             const double *__restrict__ lsrf, double *Auu,
                                                             double *Avv) {
    const int NX = nx - 1, NY = ny - 1;
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    if (q >= (long long)NX * NY) return;
    if (!active_vertex[q]) return;
    const int j = (int)(q / NX) + 1, i = (int)(q - (long long)(j - 1) * NX) + 1;  // 1-based
    auto Lf = [&](int ii, int jj) { return lsrf[(ii - 1) + (long long)nx * (jj - 1)]; };
    auto S = [&](int ii, int jj) { return (Lf(ii, jj + 1) + Lf(ii + 1, jj + 1) + Lf(ii, jj) + Lf(ii + 1, jj)) / 4.0; };
    double ddx = 0.0, ddy = 0.0;
    if (i >= 2 && i <= NX - 1 && j >= 2 && j <= NY - 1) {
        double gx[4], gy[4];  // at (i,j), (i-1,j), (i,j-1), (i-1,j-1)
        const int oi[4] = {0, -1, 0, -1}, oj[4] = {0, 0, -1, -1};
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            const int a = i + oi[n], b = j + oj[n];
            const double s00 = S(a, b), s10 = S(a + 1, b), s01 = S(a, b + 1), s11 = S(a + 1, b + 1);
            gx[n] = ((s11 - s01) / dx + (s10 - s00) / dx) / 2.0;
            gy[n] = ((s11 - s10) / dy + (s01 - s00) / dy) / 2.0;
        }
        ddx = (gx[0] + gx[1] + gx[2] + gx[3]) / 4.0;
        ddy = (gy[0] + gy[1] + gy[2] + gy[3]) / 4.0;
    }
    const double tx = atan(fabs(ddx)), ty = atan(fabs(ddy));
    const long long a = L.at(4, 0, q);
    Auu[a] = Auu[a] + (dx * dy / kAsmVol0) * bex[q] / cos(tx);
    Avv[a] = Avv[a] + (dx * dy / kAsmVol0) * bey[q] / cos(ty);
}

// ---------------------------------------------------------------------------
// assemble_stiffness_matrix_2d, L1L2 branch (:5225-5250 with compute_effective_viscosity_L1L2
// :7474-7726): per Gauss point and layer the cubic for tau_parallel (Fortran's a**3 is (a*a)*a,
// x**(1/3) is pow) and efvs = 1/(2A) for n = 1 or 1/(2A(tau_par^2 + tau_perp^2)) for n = 3 (the
// host rejects other n).  No state; the cell's own thread sums the layer viscosities over the
// points into efvs (zeroed by the host), in the reference's order, and divides by 4.
struct L1l2Args {
    const double *dsdx, *dsdy;  // (nx-1, ny-1) surface gradient at the vertices
    const double *flwa;         // (nz-1, nx, ny)
    int linear;                 // n_glen == 1
};

__device__ void asm_cell_row_l1l2(const AsmArgs &a, const L1l2Args &l, int ie, int je, int nr, bool own,
                                  double acc[4][9]) {
    const long long NX = a.nx - 1;
    const int nl = a.nz - 1;
    double x[4], y[4], u[4], v[4], h[4], sx[4], sy[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        const long long q = (long long)(ie + c_ish3[n] - 1) + NX * (je + c_jsh3[n] - 1);
        x[n] = a.xv[q];
        y[n] = a.yv[q];
        u[n] = a.u[q];
        v[n] = a.v[q];
        h[n] = a.thck[q];
        sx[n] = l.dsdx[q];
        sy[n] = l.dsdy[q];
    }
    const long long cidx = (ie - 1) + (long long)a.nx * (je - 1);
    const double *fl = l.flwa + (long long)nl * cidx, *ff = a.flwafact + (long long)nl * cidx;
    double *ecell = a.efvs + (long long)nl * cidx;
    double Kuu[4], Kuv[4], Kvu[4], Kvv[4];
#pragma unroll
    for (int nc = 0; nc < 4; ++nc) Kuu[nc] = Kuv[nc] = Kvu[nc] = Kvv[nc] = 0.0;
    for (int p = 0; p < 4; ++p) {
        const double *dxr = c_asm_ref2.dxr[p], *dyr = c_asm_ref2.dyr[p], *phi = c_asm_ref2.phi[p];
        double J00 = 0.0, J01 = 0.0, J10 = 0.0, J11 = 0.0;
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            J00 = J00 + dxr[n] * x[n];
            J01 = J01 + dxr[n] * y[n];
            J10 = J10 + dyr[n] * x[n];
            J11 = J11 + dyr[n] * y[n];
        }
        const double detJ = J00 * J11 - J01 * J10;
        if (!(fabs(detJ) > 0.0)) {
            atomicExch(a.singular, 1);
            return;
        }
        const double i00 = J11 / detJ, i01 = -J01 / detJ, i10 = -J10 / detJ, i11 = J00 / detJ;
        double dx[4], dy[4];
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            dx[n] = 0.0 + i00 * dxr[n] + i01 * dyr[n];
            dy[n] = 0.0 + i10 * dxr[n] + i11 * dyr[n];
        }
        double du_dx = 0.0, du_dy = 0.0, dv_dx = 0.0, dv_dy = 0.0, ds_dx = 0.0, ds_dy = 0.0, thck = 0.0;
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            du_dx = du_dx + dx[n] * u[n];
            du_dy = du_dy + dy[n] * u[n];
            dv_dx = dv_dx + dx[n] * v[n];
            dv_dy = dv_dy + dy[n] * v[n];
            ds_dx = ds_dx + phi[n] * sx[n];
            ds_dy = ds_dy + phi[n] * sy[n];
            thck = thck + phi[n] * h[n];
        }
        const double sh = dv_dx + du_dy;
        const double effstrain = sqrt(a.effstrain_min * a.effstrain_min + du_dx * du_dx + dv_dy * dv_dy +
                                      du_dx * dv_dy + 0.25 * (sh * sh));
        double vavg = 0.0;
        for (int k = 0; k < nl; ++k) {
            double e;
            if (a.whichefvs == 0) {
                e = a.efvs_constant;
            } else if (a.whichefvs == 1) {
                e = ff[k] * a.flowfact_pow;
            } else {
                const double depth = thck * a.sigma[k + 1];
                const double grads = sqrt(ds_dx * ds_dx + ds_dy * ds_dy);
                const double tau_perp = 910.0 * 9.81 * depth * grads;  // rhoi*grav, glimmer_physcon.F90:67,69
                const double aa = tau_perp * tau_perp;
                const double b = -effstrain / fl[k];
                const double a3 = (aa * aa) * aa;
                const double c = sqrt(b * b / 4.0 + a3 / 27.0);
                const double rootA = pow(-b / 2.0 + c, 1.0 / 3.0);
                const double rootB = (a3 / 27.0 > 1.0e-6 * (b * b / 4.0)) ? -pow(b / 2.0 + c, 1.0 / 3.0)
                                                                        : -aa / (3.0 * pow(fabs(b), 1.0 / 3.0));
                const double tp = rootA + rootB;
                e = l.linear ? 1.0 / (2.0 * fl[k]) : 1.0 / (2.0 * fl[k] * (tp * tp + tau_perp * tau_perp));
            }
            if (own) ecell[k] = ecell[k] + e;
            vavg = vavg + e * (a.sigma[k + 1] - a.sigma[k]);
        }
        double h_qp = 0.0;
#pragma unroll
        for (int n = 0; n < 4; ++n) h_qp = h_qp + phi[n] * h[n];
        const double f = h_qp * vavg * 1.0 * detJ / kAsmVol0;
        const double zero = 0.0 * 0.0;  // dphi_dz(nr)*dphi_dz(nc) of the Blatter-Pattyn form, dphi_dz = 0
#pragma unroll
        for (int nc = 0; nc < 4; ++nc) {
            Kuu[nc] = Kuu[nc] + f * (4.0 * dx[nr] * dx[nc] + dy[nr] * dy[nc] + zero);
            Kuv[nc] = Kuv[nc] + f * (2.0 * dx[nr] * dy[nc] + dy[nr] * dx[nc]);
            Kvu[nc] = Kvu[nc] + f * (2.0 * dy[nr] * dx[nc] + dx[nr] * dy[nc]);
            Kvv[nc] = Kvv[nc] + f * (4.0 * dy[nr] * dy[nc] + dx[nr] * dx[nc] + zero);
        }
    }
    if (own)
        for (int k = 0; k < nl; ++k) ecell[k] = ecell[k] / 4;
#pragma unroll
    for (int nc = 0; nc < 4; ++nc) {
        const int m = (c_ish3[nc] - c_ish3[nr] + 1) + 3 * (c_jsh3[nc] - c_jsh3[nr] + 1);
        acc[0][m] = acc[0][m] + Kuu[nc];
        acc[1][m] = acc[1][m] + Kuv[nc];
        acc[2][m] = acc[2][m] + Kvu[nc];
        acc[3][m] = acc[3][m] + Kvv[nc];
    }
}

__global__ void __launch_bounds__(kAsmBlock) k_assemble2d_l1l2(AsmArgs a, L1l2Args l, SymIdx L, double *Auu,
                                                               double *Auv, double *Avu, double *Avv) {
    const long long NX = a.nx - 1, NQ = NX * (a.ny - 1);
    const long long q = (long long)blockIdx.x * kAsmBlock + threadIdx.x;
    if (q >= NQ) return;
    const int j0 = (int)(q / NX), i0 = (int)(q - (long long)j0 * NX);
    const int iR = i0 + 1, jR = j0 + 1;
    double acc[4][9];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int c = 0; c < 9; ++c) acc[b][c] = 0.0;
    for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di) {
            const int je = jR + dj, ie = iR + di;
            if (ie < a.nhalo + 1 || ie > a.nx - a.nhalo + 1 || je < a.nhalo + 1 || je > a.ny - a.nhalo + 1) continue;
            if (!a.active_cell[(ie - 1) + (long long)a.nx * (je - 1)]) continue;
            const int nr = dj == 0 ? (di == 0 ? 2 : 3) : (di == 0 ? 1 : 0);
            asm_cell_row_l1l2(a, l, ie, je, nr, dj == 0 && di == 0, acc);
        }
    double *B[4] = {Auu, Auv, Avu, Avv};
#pragma unroll
    for (int b = 0; b < 4; ++b)
        for (int c = 0; c < 9; ++c) B[b][L.at(c, 0, q)] = acc[b][c];
}

// ---------------------------------------------------------------------------
// load_vector_gravity (:4228-4449)
// ---------------------------------------------------------------------------
// Local form (whichassemble_taud = 1, :4283-4304): one thread per vertex and level; at an active
// vertex load -= rhoi*grav*dx*dy*dz/vol0 * ds/dx with dz = stagthck*(stagwbndsigma(k) -
// stagwbndsigma(k-1)).  The loads are in the caller's (nz, nx-1, ny-1) layout or planes (W).
__global__ void __launch_bounds__(kBlock) k_load_local(int nx, int ny, int nz, double dx, double dy, VecIdx W,
                                                       const int32_t *__restrict__ active_vertex,
                                                       const double *__restrict__ stagwbndsigma,
                                                       const double *__restrict__ stagthck,
                                                       const double *__restrict__ dsdx,
                                                       const double *__restrict__ dsdy, double *loadu, double *loadv) {
    const long long NQ = (long long)(nx - 1) * (ny - 1);
    const long long t = (long long)blockIdx.x * kBlock + threadIdx.x;
    if (t >= (long long)nz * NQ) return;
    const int k = (int)(t / NQ);
    const long long q = t - (long long)k * NQ;
    if (!active_vertex[q]) return;
    const double dz = stagthck[q] * (stagwbndsigma[k + 1] - stagwbndsigma[k]);
    const long long e = W.at(k, q);
    loadu[e] = loadu[e] - 910.0 * 9.81 * dx * dy * dz / kAsmVol0 * dsdx[q];
    loadv[e] = loadv[e] - 910.0 * 9.81 * dx * dy * dz / kAsmVol0 * dsdy[q];
}

// Standard form (:4305-4447), one thread per node: the elements containing it in the reference's
// element order (as k_assemble3d), each element's 8 Gauss points (detJ as
// get_basis_function_derivatives_3d computes it, ds/dx at the point), and the node's share
// rhoi*grav*w*detJ/vol0 * (ds/dx) * phi_n subtracted point by point.
__global__ void __launch_bounds__(kAsmBlock) k_load_standard(AsmArgs a, VecIdx W, const double *__restrict__ dsdx,
                                                             const double *__restrict__ dsdy, double *loadu,
                                                             double *loadv) {
    const long long NX = a.nx - 1, NQ = NX * (a.ny - 1);
    const long long t = (long long)blockIdx.x * kAsmBlock + threadIdx.x;
    if (t >= (long long)a.nz * NQ) return;
    const int k0 = (int)(t / NQ);
    const long long q = t - (long long)k0 * NQ;
    const int j0 = (int)(q / NX), i0 = (int)(q - (long long)j0 * NX);
    const int iR = i0 + 1, jR = j0 + 1, kR = k0 + 1;
    const long long eP = W.at(k0, q);
    double lu = loadu[eP], lv = loadv[eP];
    bool any = false;
    for (int dj = 0; dj < 2; ++dj)
        for (int di = 0; di < 2; ++di)
            for (int dk = 0; dk < 2; ++dk) {
                const int je = jR + dj, ie = iR + di, ke = kR - 1 + dk;
                if (ke < 1 || ke > a.nz - 1) continue;
                if (ie < a.nhalo + 1 || ie > a.nx - a.nhalo + 1 || je < a.nhalo + 1 || je > a.ny - a.nhalo + 1)
                    continue;
                if (!a.active_cell[(ie - 1) + (long long)a.nx * (je - 1)]) continue;
                any = true;
                const int nr = (dk == 0 ? 0 : 4) + (dj == 0 ? (di == 0 ? 2 : 3) : (di == 0 ? 1 : 0));
                double x[8], y[8], z[8], sx[8], sy[8];
#pragma unroll
                for (int n = 0; n < 8; ++n) {
                    const int iN = ie + c_ish7[n], jN = je + c_jsh7[n], kN = ke + c_ksh7[n];
                    const long long qn = (long long)(iN - 1) + NX * (jN - 1);
                    x[n] = a.xv[qn];
                    y[n] = a.yv[qn];
                    z[n] = a.usrf[qn] - a.sigma[kN - 1] * a.thck[qn];
                    sx[n] = dsdx[qn];
                    sy[n] = dsdy[qn];
                }
                for (int p = 0; p < 8; ++p) {
                    const double *dxr = c_asm_ref.dxr[p], *dyr = c_asm_ref.dyr[p], *dzr = c_asm_ref.dzr[p];
                    double J00 = 0.0, J01 = 0.0, J02 = 0.0, J10 = 0.0, J11 = 0.0, J12 = 0.0, J20 = 0.0, J21 = 0.0,
                           J22 = 0.0;
#pragma unroll
                    for (int n = 0; n < 8; ++n) {
                        J00 = J00 + dxr[n] * x[n];
                        J01 = J01 + dxr[n] * y[n];
                        J02 = J02 + dxr[n] * z[n];
                        J10 = J10 + dyr[n] * x[n];
                        J11 = J11 + dyr[n] * y[n];
                        J12 = J12 + dyr[n] * z[n];
                        J20 = J20 + dzr[n] * x[n];
                        J21 = J21 + dzr[n] * y[n];
                        J22 = J22 + dzr[n] * z[n];
                    }
                    const double c00 = J11 * J22 - J12 * J21, c01 = -(J10 * J22 - J12 * J20),
                                 c02 = J10 * J21 - J11 * J20;
                    const double detJ = J00 * c00 + J01 * c01 + J02 * c02;
                    if (!(fabs(detJ) > 0.0)) {
                        atomicExch(a.singular, 1);
                        continue;
                    }
                    double sxq = 0.0, syq = 0.0;
#pragma unroll
                    for (int n = 0; n < 8; ++n) {
                        sxq = sxq + c_asm_ref.phi[p][n] * sx[n];
                        syq = syq + c_asm_ref.phi[p][n] * sy[n];
                    }
                    lu = lu - 910.0 * 9.81 * c_asm_ref.wqp[p] * detJ / kAsmVol0 * sxq * c_asm_ref.phi[p][nr];
                    lv = lv - 910.0 * 9.81 * c_asm_ref.wqp[p] * detJ / kAsmVol0 * syq * c_asm_ref.phi[p][nr];
                }
            }
    if (!any) return;
    loadu[eP] = lu;
    loadv[eP] = lv;
}

}  // namespace cismgpu
