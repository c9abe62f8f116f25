// element.cuh -- element state (TET10 / TET4) and the tiled, fused internal-force
// device code shared by the standalone force kernel and the persistent solvers.
//
// HBM layout (all device arrays owned by tlfea_element_s):
//   positions       x, y, z            FP64 SoA, mesh node order (x12/y12/z12 of
//                                      FEAT10Data.cuh:756); FP32 mode adds the
//                                      displacement u = x - X0 as FP32 SoA.
//   tiles           elements sorted along a Morton curve of their centroids and
//                   cut into tiles of TILE_ELEMS; each tile owns a sorted table
//                   of the nodes its elements touch ("local nodes").
//   grad (per tile) [tile][q][a*3+j][t]   dN_a/dx_j of tile element t at QP q
//                                      (component-major inside the tile, so a
//                                      warp's load of one component is one
//                                      contiguous 128/256-byte segment)
//   dv   (per tile) [tile][q][t]          detJ(e,q) * w_q
//   lconn(per tile) [tile][a][t]          uint16 local node of slot a
//   incidence       per local node, the (slot, element) pairs that touch it,
//                   in element-slot order: the fixed summation order of the
//                   deterministic scatter.
//   boundary        local nodes shared with other tiles write a per-tile
//                   partial; a second pass sums the partials of each shared
//                   node in tile order.  Interior nodes are written directly.
#pragma once

#include <vector>

#include "common.cuh"

namespace tlfea {

struct Tiling {
    int te = TILE_ELEMS;
    int n_tiles = 0;
    int max_local = 0;
    long long n_local_total = 0;
    int n_pslots = 0;
    int n_bnodes = 0;
    int n_orphans = 0;  // nodes touched by no element (never written by the scatter)
    int* node_off = nullptr;        // n_tiles + 1
    int* ln_gid = nullptr;          // n_local_total
    int* ln_pslot = nullptr;        // n_local_total, -1 = interior
    uint16_t* ln_inc_end = nullptr; // n_local_total, end offset in the tile's incidence
    uint16_t* inc = nullptr;        // n_tiles*te*npe: (slot << TILE_SHIFT) | element
    uint16_t* lconn = nullptr;      // n_tiles*npe*te
    int* tile_elem = nullptr;       // n_tiles*te, original element or -1 (padding)
    int* elem_slot = nullptr;       // E, tile slot of each original element
    int* bnode_gid = nullptr;       // n_bnodes
    int* bnode_off = nullptr;       // n_bnodes + 1
    int* bnode_slots = nullptr;     // n_pslots
    int* node_bidx = nullptr;       // N, boundary index or -1
    // Tile-ordered node record: every tile's local nodes in a block padded to a multiple
    // of TILE_NODE_PAD entries (so each block starts 16-byte aligned for every element
    // type and one bulk copy moves it).  pad_gid: global node (-1 = padding); pad_dst:
    // the scatter destination (global id, or -(partial slot + 1)); pad_iend: incidence
    // end; sx/sy/sz: the node values the force kernels stage (FP64 positions, or FP32
    // mode's displacements), refreshed from x (and X0) after the positions change.
    long long n_pad = 0;
    int max_local_pad = 0;
    int* pad_off = nullptr;         // n_tiles + 1, in entries
    int* pad_gid = nullptr;         // n_pad
    int* pad_dst = nullptr;         // n_pad
    uint16_t* pad_iend = nullptr;   // n_pad
    double* sx = nullptr;           // n_pad
    double* sy = nullptr;
    double* sz = nullptr;
    double* grad64 = nullptr;
    double* dv64 = nullptr;
    float* grad32 = nullptr;
    float* dv32 = nullptr;
    // J^-1 = dxi/dX per (tile, QP), [tile][q][3 * k + j][TILE_ELEMS]: the
    // compact geometry stream (9 values instead of 3 * NPE gradients)
    double* ji64 = nullptr;
    float* ji32 = nullptr;
    double* partial64 = nullptr;
    float* partial32 = nullptr;
    std::vector<int> h_tile_elem;  // host copy of tile_elem
};

// Per-call arguments of the tile routine.
// Barycentric coordinates L = (1 - xi - eta - zeta, xi, eta, zeta) of the
// quadrature points, the only per-QP data the compact geometry stream needs.
struct QpBary {
    double L[5][4];
};

template <typename R>
struct TileArgs {
    const int* node_off;
    const int* ln_gid;
    const int* ln_pslot;
    const uint16_t* ln_inc_end;
    const uint16_t* inc;
    const uint16_t* lconn;
    const int* tile_elem;
    const R* grad;
    const R* ji;  // J^-1 per (tile, QP), the compact geometry stream
    const R* dv;
    const R* px;  // FP64 mode: positions x (null in FP32 mode)
    const R* py;
    const R* pz;
    // FP32 mode: each tile stages its nodes' FP64 displacements (stage_pos), from the
    // interleaved record u64 = x - X0 when it is given, else from the FP64 positions and
    // reference positions
    const double* u64;
    const double* x64;
    const double* y64;
    const double* z64;
    const double* X0x;
    const double* X0y;
    const double* X0z;
    const double* v;  // interleaved velocities for the Kelvin-Voigt term, or null
    double* Pst;      // stored P in the reference layout (CalcP / CalcInternalForce)
    R* f_out;         // interleaved 3N
    R* partial;       // 3 * n_pslots
    R lambda, mu, eta, lamd;
    double mu10, mu01, kappa;  // Mooney-Rivlin (MR instantiations)
    const double* vp;          // MASS instantiations: previous-step velocity (interleaved 3N)
    double mass_scale;         // MASS instantiations: rho / dt
    int max_local;
    // the tile-ordered node record (Tiling::pad_*), read by bulk copies
    const int* pad_off;
    const int* pad_dst;
    const uint16_t* pad_iend;
    const int* pad_gid;
    const double* sx;
    const double* sy;
    const double* sz;
    QpBary qb;
};

// Offset of gradient (node a, component j) of the element in lane t within one QP
// slice of the gradient stream.  FP64: component-major [a*3 + j][t].  FP32: node
// pairs interleaved, [(a/2)*3 + j][t][a%2], so that one 8-byte shared-memory load
// gives (gradN_a, gradN_(a+1)) for the paired FP32 arithmetic of the force kernel
// (NPE is even: 10 or 4).
template <typename R>
__host__ __device__ __forceinline__ size_t grad_slot(int a, int j, int t) {
    if constexpr (sizeof(R) == 4)
        return ((size_t)((a >> 1) * 3 + j) * TILE_ELEMS + t) * 2 + (a & 1);
    else
        return (size_t)(a * 3 + j) * TILE_ELEMS + t;
}

// Node values staged for a tile, always FP64 in shared memory.  FP64 mode: the
// positions themselves (F = sum_a x_a (x) gradN_a, the reference's formula).  FP32
// mode: the displacements u = x - X0, from the interleaved FP64 record u64 when it is
// given, else differenced from the FP64 positions and reference positions.
template <typename R>
__device__ __forceinline__ void stage_pos(const TileArgs<R>& A, int gid, double& x, double& y, double& z) {
    if constexpr (sizeof(R) == 4) {
        if (A.u64) {
            x = A.u64[3 * gid + 0];
            y = A.u64[3 * gid + 1];
            z = A.u64[3 * gid + 2];
        } else {
            x = A.x64[gid] - A.X0x[gid];
            y = A.y64[gid] - A.X0y[gid];
            z = A.z64[gid] - A.X0z[gid];
        }
    } else {
        x = A.px[gid];
        y = A.py[gid];
        z = A.pz[gid];
    }
}

// One element's node values for the force arithmetic, from the tile's staged FP64
// values (xs/ys/zs, or interleaved for `element_velocities`).  FP64 mode: the values
// as staged.  FP32 mode: relative to the element's first node, differenced in FP64
// and rounded once, u_a - u_0.  The shape-function gradients sum to zero, so
// H = sum_a (u_a - u_0) (x) gradN_a exactly; both roundings -- of the node values and
// of the FP32 gradients -- then scale with how much u varies across the element
// instead of with |u|, which keeps the FP32 force accurate at large displacements
// and rotations.
template <typename R, int NPE>
__device__ __forceinline__ void element_nodes(const double* xs, const double* ys, const double* zs, const int* lc,
                                              R xa[NPE][3]) {
    double b0 = 0.0, b1 = 0.0, b2 = 0.0;
    if constexpr (sizeof(R) == 4) {
        b0 = xs[lc[0]];
        b1 = ys[lc[0]];
        b2 = zs[lc[0]];
    }
#pragma unroll
    for (int a = 0; a < NPE; ++a) {
        xa[a][0] = R(xs[lc[a]] - b0);
        xa[a][1] = R(ys[lc[a]] - b1);
        xa[a][2] = R(zs[lc[a]] - b2);
    }
}

template <typename R, int NPE>
__device__ __forceinline__ void element_velocities(const double* vs, const int* lc, R va[NPE][3]) {
    double b[3] = {0.0, 0.0, 0.0};
    if constexpr (sizeof(R) == 4) {
#pragma unroll
        for (int d = 0; d < 3; ++d) b[d] = vs[3 * lc[0] + d];
    }
#pragma unroll
    for (int a = 0; a < NPE; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) va[a][d] = R(vs[3 * lc[a] + d] - b[d]);
}

// Tile routine modes.
enum { TILE_FORCE = 0, TILE_STORE_P = 1, TILE_FORCE_FROM_P = 2 };


// ----------------------------------------------------------------------------
// Compact geometry: with J^-1 = dxi/dX stored per QP, gradN_a = J^-T dN_a/dxi and
//   F (or H) = sum_a x_a (x) gradN_a = G J^-1,      G = dx/dxi = sum_a x_a (x) dN_a/dxi,
//   f_a += dV P gradN_a = Q dN_a/dxi,               Q = dV P J^-T,
// and for the tetrahedra of the reference node order (corners 0..3, edge nodes
// 4..9 on (0,1) (1,2) (0,2) (0,3) (1,3) (2,3)) both sums follow the barycentric
// structure of the shape functions (corner N_i = L_i (2 L_i - 1), edge
// N_ij = 4 L_i L_j, dL_0/dxi_k = -1, dL_(k+1)/dxi_k = 1):
//   y_i = dx/dL_i = (4 L_i - 1) x_i + 4 sum_(j != i) L_j x_ij,  G[:, k] = y_(k+1) - y_0,
//   r_0 = -(Q[:,0] + Q[:,1] + Q[:,2]), r_(k+1) = Q[:, k],
//   f_i += (4 L_i - 1) r_i,  f_ij += 4 (L_i r_j + L_j r_i).
// The same F and forces as the per-node gradients, from 9 stored values per QP
// instead of 3 * NPE.
// ----------------------------------------------------------------------------

// G[d][k] = dx_d/dxi_k from the nodal values xa[a][d].
template <typename R, int NPE>
__device__ __forceinline__ void tet_dx_dxi(const R (&xa)[NPE][3], const R L[4], R G[3][3]) {
    if constexpr (NPE == 10) {
        const R c0 = R(4) * L[0] - R(1), c1 = R(4) * L[1] - R(1), c2 = R(4) * L[2] - R(1), c3 = R(4) * L[3] - R(1);
        const R l0 = R(4) * L[0], l1 = R(4) * L[1], l2 = R(4) * L[2], l3 = R(4) * L[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const R y0 = c0 * xa[0][d] + l1 * xa[4][d] + l2 * xa[6][d] + l3 * xa[7][d];
            const R y1 = c1 * xa[1][d] + l0 * xa[4][d] + l2 * xa[5][d] + l3 * xa[8][d];
            const R y2 = c2 * xa[2][d] + l1 * xa[5][d] + l0 * xa[6][d] + l3 * xa[9][d];
            const R y3 = c3 * xa[3][d] + l0 * xa[7][d] + l1 * xa[8][d] + l2 * xa[9][d];
            G[d][0] = y1 - y0;
            G[d][1] = y2 - y0;
            G[d][2] = y3 - y0;
        }
    } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            G[d][0] = xa[1][d] - xa[0][d];
            G[d][1] = xa[2][d] - xa[0][d];
            G[d][2] = xa[3][d] - xa[0][d];
        }
    }
}

// The same dx/dxi with the node values read through x(a, d) where they are used (from
// shared memory, say), so they need not be held in registers all at once.
template <typename R, int NPE, typename X>
__device__ __forceinline__ void tet_dx_dxi_at(X x, const R L[4], R G[3][3]) {
    if constexpr (NPE == 10) {
        const R c0 = R(4) * L[0] - R(1), c1 = R(4) * L[1] - R(1), c2 = R(4) * L[2] - R(1), c3 = R(4) * L[3] - R(1);
        const R l0 = R(4) * L[0], l1 = R(4) * L[1], l2 = R(4) * L[2], l3 = R(4) * L[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const R y0 = c0 * x(0, d) + l1 * x(4, d) + l2 * x(6, d) + l3 * x(7, d);
            const R y1 = c1 * x(1, d) + l0 * x(4, d) + l2 * x(5, d) + l3 * x(8, d);
            const R y2 = c2 * x(2, d) + l1 * x(5, d) + l0 * x(6, d) + l3 * x(9, d);
            const R y3 = c3 * x(3, d) + l0 * x(7, d) + l1 * x(8, d) + l2 * x(9, d);
            G[d][0] = y1 - y0;
            G[d][1] = y2 - y0;
            G[d][2] = y3 - y0;
        }
    } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const R x0 = x(0, d);
            G[d][0] = x(1, d) - x0;
            G[d][1] = x(2, d) - x0;
            G[d][2] = x(3, d) - x0;
        }
    }
}

// acc(a, d, Q[d][:] . dN_a/dxi) for every node a and component d.
template <typename R, int NPE, typename Acc>
__device__ __forceinline__ void tet_scatter(const R Q[3][3], const R L[4], Acc acc) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const R r0 = -(Q[d][0] + Q[d][1] + Q[d][2]), r1 = Q[d][0], r2 = Q[d][1], r3 = Q[d][2];
        if constexpr (NPE == 10) {
            const R l0 = R(4) * L[0], l1 = R(4) * L[1], l2 = R(4) * L[2], l3 = R(4) * L[3];
            acc(0, d, (l0 - R(1)) * r0);
            acc(1, d, (l1 - R(1)) * r1);
            acc(2, d, (l2 - R(1)) * r2);
            acc(3, d, (l3 - R(1)) * r3);
            acc(4, d, l0 * r1 + l1 * r0);
            acc(5, d, l1 * r2 + l2 * r1);
            acc(6, d, l0 * r2 + l2 * r0);
            acc(7, d, l0 * r3 + l3 * r0);
            acc(8, d, l1 * r3 + l3 * r1);
            acc(9, d, l2 * r3 + l3 * r2);
        } else {
            acc(0, d, r0);
            acc(1, d, r1);
            acc(2, d, r2);
            acc(3, d, r3);
        }
    }
}

// M J^-1 (ji row-major J^-1) and M J^-T.
template <typename R>
__device__ __forceinline__ void mul_jinv(const R M[3][3], const R ji[9], R out[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) out[i][j] = M[i][0] * ji[j] + M[i][1] * ji[3 + j] + M[i][2] * ji[6 + j];
}
template <typename R>
__device__ __forceinline__ void mul_jinv_t(const R M[3][3], const R ji[9], R out[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            out[i][k] = M[i][0] * ji[3 * k] + M[i][1] * ji[3 * k + 1] + M[i][2] * ji[3 * k + 2];
}

template <typename R>
__device__ __forceinline__ R ld_stream(const R* p) {
    return __ldcs(p);
}

// P from F for the SVK law in the reference's form
// lambda*(tr(F^T F)/2 - 3/2) F + mu (F F^T F - F)  (SVK.cuh:17-39, FEAT10DataFunc.cuh:233-281).
__device__ __forceinline__ void svk_p_reference(const double F[3][3], double lambda, double mu, double P[3][3]) {
    double FtF[3][3], FFt[3][3], FFtF[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) s += F[k][i] * F[k][j];
            FtF[i][j] = s;
        }
    const double tr = FtF[0][0] + FtF[1][1] + FtF[2][2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) s += F[i][k] * F[j][k];
            FFt[i][j] = s;
        }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) s += FFt[i][k] * F[k][j];
            FFtF[i][j] = s;
        }
    const double lf = lambda * (0.5 * tr - 1.5);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) P[i][j] = lf * F[i][j] + mu * (FFtF[i][j] - F[i][j]);
}

// Kelvin-Voigt P_vis = F (2 eta Edot + lamd tr(Edot) I), Edot = (Fdot^T F + F^T Fdot)/2
// (FEAT10DataFunc.cuh:135-222).
template <typename R>
__device__ __forceinline__ void kelvin_voigt(const R F[3][3], const R Fd[3][3], R eta, R lamd, R Pv[3][3]) {
    R Ed[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            R a = R(0), b = R(0);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                a += Fd[k][i] * F[k][j];
                b += F[k][i] * Fd[k][j];
            }
            Ed[i][j] = R(0.5) * (a + b);
        }
    const R tr = Ed[0][0] + Ed[1][1] + Ed[2][2];
    R S[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) S[i][j] = R(2) * eta * Ed[i][j] + lamd * tr * (i == j ? R(1) : R(0));
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            R s = R(0);
#pragma unroll
            for (int k = 0; k < 3; ++k) s += F[i][k] * S[k][j];
            Pv[i][j] = s;
        }
}

// One tile: stage the tile's nodes in shared memory, evaluate its elements (one
// thread per element, QP by QP, gradients streamed from HBM), reduce element
// forces per node in the fixed incidence order, write interior nodes and
// boundary partials.  Must be called by all TILE_ELEMS threads of the block.
//
// R = double: F = sum_a x_a (x) gradN_a and the reference SVK formula.
// R = float : the FP32 mode.  F = I + H with H = sum_a u_a (x) gradN_a from
//             the FP32 displacement, and P = (I + H) S, S = lambda tr(E) I + 2 mu E,
//             E = (H + H^T + H^T H)/2 -- algebraically the same SVK stress,
//             without the cancellation of tr(F^T F) - 3 near F = I.
// Mooney-Rivlin first Piola stress (mr_compute_P, MooneyRivlin.cuh:46-104), FP64:
// C = F^T F, I1 = tr C, I2 = (I1^2 - tr C^2) / 2, J = det F, F^-T by cofactors
// with |J| clamped to 1e-12 for the inverse, and
// P = 2 mu10 J^-2/3 (F - I1/3 F^-T) + 2 mu01 J^-4/3 (I1 F - F C - 2 I2/3 F^-T)
//   + kappa (J - 1) J F^-T.
__device__ __forceinline__ void mooney_rivlin_p(const double F[3][3], double mu10, double mu01, double kappa,
                                                double P[3][3]) {
    double C[3][3], FC[3][3], FiT[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C[i][j] = F[0][i] * F[0][j] + F[1][i] * F[1][j] + F[2][i] * F[2][j];
    const double I1 = C[0][0] + C[1][1] + C[2][2];
    double trC2 = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) trC2 += C[i][k] * C[k][i];
    const double I2 = 0.5 * (I1 * I1 - trC2);
    const double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                     F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                     F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
    const double dj = (fabs(J) < 1e-12) ? ((J >= 0.0) ? 1e-12 : -1e-12) : J;
    const double id = 1.0 / dj;
    FiT[0][0] = (F[1][1] * F[2][2] - F[1][2] * F[2][1]) * id;
    FiT[0][1] = (F[1][2] * F[2][0] - F[1][0] * F[2][2]) * id;
    FiT[0][2] = (F[1][0] * F[2][1] - F[1][1] * F[2][0]) * id;
    FiT[1][0] = (F[0][2] * F[2][1] - F[0][1] * F[2][2]) * id;
    FiT[1][1] = (F[0][0] * F[2][2] - F[0][2] * F[2][0]) * id;
    FiT[1][2] = (F[0][1] * F[2][0] - F[0][0] * F[2][1]) * id;
    FiT[2][0] = (F[0][1] * F[1][2] - F[0][2] * F[1][1]) * id;
    FiT[2][1] = (F[0][2] * F[1][0] - F[0][0] * F[1][2]) * id;
    FiT[2][2] = (F[0][0] * F[1][1] - F[0][1] * F[1][0]) * id;
    const double j13 = cbrt(J);
    const double jm23 = 1.0 / (j13 * j13), jm43 = jm23 * jm23;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) FC[i][j] = F[i][0] * C[0][j] + F[i][1] * C[1][j] + F[i][2] * C[2][j];
    const double t1 = 2.0 * mu10 * jm23, t2 = 2.0 * mu01 * jm43, t3 = kappa * (J - 1.0) * J;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            P[i][j] = t1 * (F[i][j] - (I1 / 3.0) * FiT[i][j]) +
                      t2 * (I1 * F[i][j] - FC[i][j] - (2.0 * I2 / 3.0) * FiT[i][j]) + t3 * FiT[i][j];
}

// Mooney-Rivlin consistent tangent A_ijkl = dP_ij / dF_kl (mr_compute_tangent_tensor,
// MooneyRivlin.cuh:106-221: the exact derivative of mooney_rivlin_p, term by
// term), contracted with node a's gradient: B[i][k][l] = sum_j A_ijkl ga[j], so
// the (a, b) stiffness block is K[i][k] = sum_l B[i][k][l] gb[l] dV.
__device__ __forceinline__ void mooney_rivlin_tangent_a(const double F[3][3], double mu10, double mu01, double kappa,
                                                        const double ga[3], double B[3][3][3]) {
    double C[3][3], FC[3][3], FFT[3][3], FiT[3][3], T1[3][3], T2[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            C[i][j] = F[0][i] * F[0][j] + F[1][i] * F[1][j] + F[2][i] * F[2][j];
            FFT[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
        }
    const double I1 = C[0][0] + C[1][1] + C[2][2];
    double trC2 = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) trC2 += C[i][k] * C[k][i];
    const double I2 = 0.5 * (I1 * I1 - trC2);
    const double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                     F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                     F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
    const double dj = (fabs(J) < 1e-12) ? ((J >= 0.0) ? 1e-12 : -1e-12) : J;
    const double id = 1.0 / dj;
    FiT[0][0] = (F[1][1] * F[2][2] - F[1][2] * F[2][1]) * id;
    FiT[0][1] = (F[1][2] * F[2][0] - F[1][0] * F[2][2]) * id;
    FiT[0][2] = (F[1][0] * F[2][1] - F[1][1] * F[2][0]) * id;
    FiT[1][0] = (F[0][2] * F[2][1] - F[0][1] * F[2][2]) * id;
    FiT[1][1] = (F[0][0] * F[2][2] - F[0][2] * F[2][0]) * id;
    FiT[1][2] = (F[0][1] * F[2][0] - F[0][0] * F[2][1]) * id;
    FiT[2][0] = (F[0][1] * F[1][2] - F[0][2] * F[1][1]) * id;
    FiT[2][1] = (F[0][2] * F[1][0] - F[0][0] * F[1][2]) * id;
    FiT[2][2] = (F[0][0] * F[1][1] - F[0][1] * F[1][0]) * id;
    const double j13 = cbrt(J);
    const double jm23 = 1.0 / (j13 * j13), jm43 = jm23 * jm23;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) FC[i][j] = F[i][0] * C[0][j] + F[i][1] * C[1][j] + F[i][2] * C[2][j];
    const double t1 = 2.0 * mu10 * jm23, t2 = 2.0 * mu01 * jm43, t3 = kappa * (J - 1.0) * J;
    const double dt3c = kappa * (2.0 * J - 1.0) * J;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T1[i][j] = F[i][j] - (I1 / 3.0) * FiT[i][j];
            T2[i][j] = I1 * F[i][j] - FC[i][j] - (2.0 * I2 / 3.0) * FiT[i][j];
        }
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) {
                double s = 0.0;
                for (int j = 0; j < 3; ++j) {
                    const double dik = (i == k) ? 1.0 : 0.0, djl = (j == l) ? 1.0 : 0.0;
                    const double dFiT = -FiT[i][l] * FiT[k][j];
                    const double dT1 = dik * djl - (2.0 / 3.0) * F[k][l] * FiT[i][j] + (I1 / 3.0) * FiT[i][l] * FiT[k][j];
                    const double dT2 = 2.0 * F[k][l] * F[i][j] + I1 * dik * djl -
                                       (dik * C[l][j] + F[i][l] * F[k][j] + djl * FFT[i][k]) -
                                       (4.0 / 3.0) * (I1 * F[k][l] - FC[k][l]) * FiT[i][j] +
                                       (2.0 * I2 / 3.0) * FiT[i][l] * FiT[k][j];
                    const double A = (-2.0 / 3.0) * t1 * FiT[k][l] * T1[i][j] + t1 * dT1 +
                                     (-4.0 / 3.0) * t2 * FiT[k][l] * T2[i][j] + t2 * dT2 + dt3c * FiT[k][l] * FiT[i][j] +
                                     t3 * dFiT;
                    s += A * ga[j];
                }
                B[i][k][l] = s;
            }
}

// First Piola stress of one QP from the compact-geometry gradient: FP64 takes
// F itself (the reference's SVK form), FP32 the displacement gradient H (F =
// I + H, the cancellation-free form); with DAMP the Kelvin-Voigt term of the
// velocity gradient Fd is added.
template <typename R, bool DAMP, bool MR = false>
__device__ __forceinline__ void tile_stress(const R H[3][3], const R Fd[3][3], const TileArgs<R>& A, R P[3][3],
                                            R lam, R mu) {
    if constexpr (MR) {
        // Mooney-Rivlin in FP64 whatever R is (FP32 mode: F = I + H formed in FP64)
        double F64[3][3], P64[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                F64[i][j] = (sizeof(R) == 8) ? double(H[i][j]) : double(H[i][j]) + (i == j ? 1.0 : 0.0);
        mooney_rivlin_p(F64, A.mu10, A.mu01, A.kappa, P64);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) P[i][j] = R(P64[i][j]);
    } else if constexpr (sizeof(R) == 8) {
        svk_p_reference(H, lam, mu, P);
    } else {
        R Em[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                R sm = H[i][j] + H[j][i];
#pragma unroll
                for (int k = 0; k < 3; ++k) sm += H[k][i] * H[k][j];
                Em[i][j] = R(0.5) * sm;
            }
        const R trE = Em[0][0] + Em[1][1] + Em[2][2];
        R Sm[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) Sm[i][j] = R(2) * mu * Em[i][j] + (i == j ? lam * trE : R(0));
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                R sm = Sm[i][j];
#pragma unroll
                for (int k = 0; k < 3; ++k) sm += H[i][k] * Sm[k][j];
                P[i][j] = sm;
            }
    }
    if constexpr (DAMP) {
        R F[3][3], Pv[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) F[i][j] = (sizeof(R) == 8) ? H[i][j] : H[i][j] + (i == j ? R(1) : R(0));
        kelvin_voigt<R>(F, Fd, A.eta, A.lamd, Pv);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) P[i][j] += Pv[i][j];
    }
}

// One QP of the compact-geometry force: F (or H) = (dx/dxi) J^-1 from the
// nodal values xa, the stress, and f_a (+)= (dV P J^-T) dN_a/dxi.
// Shape-function values at barycentric L (reference node order): corners
// L_i (2 L_i - 1), edges 4 L_i L_j; TET4 N_a = L_a.
template <typename R, int NPE>
__device__ __forceinline__ void tet_shape(const R L[4], R N[NPE]) {
    if constexpr (NPE == 10) {
#pragma unroll
        for (int i = 0; i < 4; ++i) N[i] = L[i] * (R(2) * L[i] - R(1));
        N[4] = R(4) * L[0] * L[1];
        N[5] = R(4) * L[1] * L[2];
        N[6] = R(4) * L[0] * L[2];
        N[7] = R(4) * L[0] * L[3];
        N[8] = R(4) * L[1] * L[3];
        N[9] = R(4) * L[2] * L[3];
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) N[i] = L[i];
    }
}

// The element's share of M (v - v_prev) / dt at one QP, added to the nodal
// forces: f_a += N_a dV w(q), w(q) = sum_b N_b w_b with w_b = rho (v_b - vp_b) / dt
// (the consistent mass M_ab = sum_q rho N_a N_b dV_q, FEAT10Data.cu:200-271,
// applied element by element instead of as an assembled row pass).
template <typename R, int NPE>
__device__ __forceinline__ void mass_qp(const R (&wa)[NPE][3], const R Lq[4], R dv, R (&f)[NPE][3]) {
    R N[NPE];
    tet_shape<R, NPE>(Lq, N);
    R w[3] = {R(0), R(0), R(0)};
#pragma unroll
    for (int b = 0; b < NPE; ++b)
#pragma unroll
        for (int d = 0; d < 3; ++d) w[d] += N[b] * wa[b][d];
#pragma unroll
    for (int a = 0; a < NPE; ++a) {
        const R s = N[a] * dv;
#pragma unroll
        for (int d = 0; d < 3; ++d) f[a][d] += s * w[d];
    }
}

template <typename R, int NPE, bool DAMP, bool FIRST, bool MR = false>
__device__ __forceinline__ void compact_qp(const TileArgs<R>& A, const R (&xa)[NPE][3], const R (&va)[NPE][3],
                                           const R ji[9], R dv, const R Lq[4], R (&f)[NPE][3], R lam, R mu) {
    R Gx[3][3], H[3][3], Fd[3][3], P[3][3], Q[3][3];
    tet_dx_dxi<R, NPE>(xa, Lq, Gx);
    mul_jinv(Gx, ji, H);
    if constexpr (DAMP) {
        R Gv[3][3];
        tet_dx_dxi<R, NPE>(va, Lq, Gv);
        mul_jinv(Gv, ji, Fd);
    }
    tile_stress<R, DAMP, MR>(H, Fd, A, P, lam, mu);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) P[i][j] *= dv;
    mul_jinv_t(P, ji, Q);
    if constexpr (FIRST)
        tet_scatter<R, NPE>(Q, Lq, [&](int a, int d, R v) { f[a][d] = v; });
    else
        tet_scatter<R, NPE>(Q, Lq, [&](int a, int d, R v) { f[a][d] += v; });
}

// Per-sequence arrays and material of the batched dynamics (FP64): process_tile with
// SEQ reads these instead of A's, so A itself stays an unmodified kernel parameter.
template <typename R>
struct TileSeq {
    const double *px, *py, *pz;  // positions
    const double *v, *vp;        // velocities (the mass term's v and v_prev; v also for damping)
    R* f_out;
    R* partial;
    R lambda, mu;
};

// MASS (force mode only): the element-wise mass term M (v - v_prev) / dt of the
// first-order solvers' gradient is added to the nodal forces (see mass_qp).
template <typename R, int NPE, int NQP, int MODE, bool DAMP, bool MR = false, bool MASS = false, bool SEQ = false>
__device__ __forceinline__ void process_tile(const TileArgs<R>& A, int tile, unsigned char* smem_raw,
                                             const TileSeq<R>* sq = nullptr) {
    static_assert(!SEQ || (sizeof(R) == 8 && MODE == TILE_FORCE), "per-sequence override: FP64 forces only");
    constexpr int TE = TILE_ELEMS;
    const int t = threadIdx.x;
    const R lam = SEQ ? sq->lambda : A.lambda, mu = SEQ ? sq->mu : A.mu;
    const double* vsrc = SEQ ? sq->v : A.v;
    const double* vpsrc = SEQ ? sq->vp : A.vp;
    // [x y z (FP64)][velocities (FP64, DAMP)][mass term (MASS)][element forces]
    double* xs = reinterpret_cast<double*>(smem_raw);
    double* ys = xs + A.max_local;
    double* zs = ys + A.max_local;
    double* vs = zs + A.max_local;
    R* ws = reinterpret_cast<R*>(DAMP ? vs + 3 * A.max_local : vs);
    R* fe = MASS ? ws + 3 * A.max_local : ws;

    const int lb = A.node_off[tile];
    const int nl = A.node_off[tile + 1] - lb;
    if (MODE == TILE_FORCE && t == 0) {
        // the tile's J^-1 and dV stream (every QP) into L2 while the node values are
        // staged, so the per-QP loads below hit L2 instead of each waiting on DRAM
        // (16-byte aligned, sizes multiples of 16 bytes)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(A.ji + (size_t)tile * NQP * 9 * TE),
                     "r"((uint32_t)(NQP * 9 * TE * sizeof(R)))
                     : "memory");
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(A.dv + (size_t)tile * NQP * TE),
                     "r"((uint32_t)(NQP * TE * sizeof(R)))
                     : "memory");
    }
    if (MODE != TILE_FORCE_FROM_P) {
#pragma unroll 4
        for (int ln = t; ln < nl; ln += TE) {  // unrolled: several nodes' gathers in flight at once
            const int gid = A.ln_gid[lb + ln];
            if constexpr (SEQ) {
                xs[ln] = sq->px[gid];
                ys[ln] = sq->py[gid];
                zs[ln] = sq->pz[gid];
            } else {
                stage_pos(A, gid, xs[ln], ys[ln], zs[ln]);
            }
            if (DAMP) {
                vs[3 * ln + 0] = vsrc[3 * gid + 0];
                vs[3 * ln + 1] = vsrc[3 * gid + 1];
                vs[3 * ln + 2] = vsrc[3 * gid + 2];
            }
            if (MASS) {
#pragma unroll
                for (int d = 0; d < 3; ++d) ws[3 * ln + d] = R((vsrc[3 * gid + d] - vpsrc[3 * gid + d]) * A.mass_scale);
            }
        }
    }
    int lc[NPE];
#pragma unroll
    for (int a = 0; a < NPE; ++a) lc[a] = A.lconn[((size_t)tile * NPE + a) * TE + t];
    const int eo = (MODE == TILE_FORCE) ? 0 : A.tile_elem[(size_t)tile * TE + t];
    __syncthreads();

    R f[NPE][3];
#pragma unroll
    for (int a = 0; a < NPE; ++a) f[a][0] = f[a][1] = f[a][2] = R(0);
    // the element's node values: FP32 reads them once per tile (element-relative, so
    // the FP64 differences are taken once); FP64 re-reads them per QP (registers)
    R xa[NPE][3], va[NPE][3];

#pragma unroll 1
    for (int q = 0; q < NQP && MODE == TILE_FORCE; ++q) {
        // the force alone: compact geometry stream (J^-1 and dV per QP)
        const R* jp = A.ji + ((size_t)tile * NQP + q) * 9 * TE + t;
        R ji[9];
#pragma unroll
        for (int m = 0; m < 9; ++m) ji[m] = ld_stream(jp + m * TE);
        const R dv = ld_stream(A.dv + ((size_t)tile * NQP + q) * TE + t);
        const R Lq[4] = {R(A.qb.L[q][0]), R(A.qb.L[q][1]), R(A.qb.L[q][2]), R(A.qb.L[q][3])};
        if (q == 0 || sizeof(R) == 8) {
            element_nodes<R, NPE>(xs, ys, zs, lc, xa);
            if (DAMP) element_velocities<R, NPE>(vs, lc, va);
        }
        compact_qp<R, NPE, DAMP, false, MR>(A, xa, va, ji, dv, Lq, f, lam, mu);
        if constexpr (MASS) {
            R wa[NPE][3];
#pragma unroll
            for (int a = 0; a < NPE; ++a)
#pragma unroll
                for (int d = 0; d < 3; ++d) wa[a][d] = ws[3 * lc[a] + d];
            mass_qp<R, NPE>(wa, Lq, dv, f);
        }
    }
#pragma unroll 1
    for (int q = 0; q < NQP && MODE != TILE_FORCE; ++q) {
        const R* gp = A.grad + ((size_t)tile * NQP + q) * (NPE * 3) * TE;
        R g[NPE][3];
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
            for (int j = 0; j < 3; ++j) g[a][j] = ld_stream(gp + grad_slot<R>(a, j, t));
        const R dv = ld_stream(A.dv + ((size_t)tile * NQP + q) * TE + t);

        R P[3][3];
        if constexpr (MODE == TILE_FORCE_FROM_P) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    P[i][j] = (eo >= 0) ? R(A.Pst[((size_t)eo * NQP + q) * 9 + i + 3 * j]) : R(0);
        } else {
            // F (FP64) or H (FP32) from the gradients, the velocity gradient for
            // the Kelvin-Voigt term, then the material law
            R H[3][3], Fd[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) H[i][j] = Fd[i][j] = R(0);
            if (q == 0 || sizeof(R) == 8) {
                element_nodes<R, NPE>(xs, ys, zs, lc, xa);
                if (DAMP) element_velocities<R, NPE>(vs, lc, va);
            }
#pragma unroll
            for (int a = 0; a < NPE; ++a)
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) H[i][j] += xa[a][i] * g[a][j];
            if (DAMP) {
#pragma unroll
                for (int a = 0; a < NPE; ++a)
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) Fd[i][j] += va[a][i] * g[a][j];
            }
            tile_stress<R, DAMP, MR>(H, Fd, A, P, lam, mu);
        }

        if constexpr (MODE == TILE_STORE_P) {
            if (eo >= 0) {
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) A.Pst[((size_t)eo * NQP + q) * 9 + i + 3 * j] = double(P[i][j]);
            }
        } else {
            // f_a += (P grad_a) dV   (FEAT10DataFunc.cuh:417-449)
#pragma unroll
            for (int a = 0; a < NPE; ++a)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    R fc = R(0);
#pragma unroll
                    for (int j = 0; j < 3; ++j) fc += P[i][j] * g[a][j];
                    f[a][i] += fc * dv;
                }
        }
    }
    if constexpr (MODE != TILE_STORE_P) {

#pragma unroll
    for (int a = 0; a < NPE; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) fe[(a * 3 + d) * TE + t] = f[a][d];
    __syncthreads();

    const uint16_t* inc = A.inc + (size_t)tile * TE * NPE;
    R* const f_out = SEQ ? sq->f_out : A.f_out;
    R* const part = SEQ ? sq->partial : A.partial;
    for (int ln = t; ln < nl; ln += TE) {
        const int beg = ln ? A.ln_inc_end[lb + ln - 1] : 0;
        const int end = A.ln_inc_end[lb + ln];
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;  // node sums in FP64 (near equilibrium they cancel)
        for (int k = beg; k < end; ++k) {
            const int ent = inc[k];
            const int base = (ent >> TILE_SHIFT) * 3 * TE + (ent & (TE - 1));
            s0 += fe[base];
            s1 += fe[base + TE];
            s2 += fe[base + 2 * TE];
        }
        const int ps = A.ln_pslot[lb + ln];
        if (ps < 0) {
            const int gid = A.ln_gid[lb + ln];
            if (MODE == TILE_FORCE_FROM_P) {
                f_out[3 * gid + 0] += s0;
                f_out[3 * gid + 1] += s1;
                f_out[3 * gid + 2] += s2;
            } else {
                f_out[3 * gid + 0] = s0;
                f_out[3 * gid + 1] = s1;
                f_out[3 * gid + 2] = s2;
            }
        } else {
            part[3 * ps + 0] = s0;
            part[3 * ps + 1] = s1;
            part[3 * ps + 2] = s2;
        }
    }
    }  // MODE != TILE_STORE_P
}

// Shared memory bytes of one tile block.
template <typename R>
inline size_t tile_smem_bytes(int npe, int max_local, bool damp, bool mass = false) {
    return sizeof(double) * (size_t)max_local * (3 + (damp ? 3 : 0)) +
           sizeof(R) * ((size_t)max_local * (mass ? 3 : 0) + (size_t)3 * npe * TILE_ELEMS);
}

}  // namespace tlfea

// ---------------------------------------------------------------- element state
struct tlfea_element_s {
    int type = TLFEA_TYPE_T10;
    int npe = tlfea::T10_NPE;
    int nqp = tlfea::T10_NQP;
    int E = 0;
    int N = 0;
    int device = 0;
    cudaStream_t stream = 0;
    bool own_stream = false;
    bool blocking = true;

    bool is_setup = false;
    bool precomputed = false;
    bool constraints_setup = false;
    bool mass_setup = false;
    bool jt_setup = false;
    bool j_setup = false;

    std::vector<int> conn;  // column-major, original element order
    std::vector<int> elem_group;  // optional tiling group per element (batch instance), set before setup
    double qx[5] = {0}, qy[5] = {0}, qz[5] = {0}, qw[5] = {0};

    double rho = 0, E_mod = 0, nu = 0, mu = 0, lambda = 0, eta_d = 0, lambda_d = 0;
    int material = TLFEA_MATERIAL_SVK;
    double mu10 = 0, mu01 = 0, kappa = 0;
    int precision = TLFEA_PRECISION_FP64;

    double *x = nullptr, *y = nullptr, *z = nullptr;
    double *xj = nullptr, *yj = nullptr, *zj = nullptr;
    double *X0x = nullptr, *X0y = nullptr, *X0z = nullptr;
    double* u64 = nullptr;  // interleaved x - X0 for the FP32 force (refreshed when positions change)
    bool u_dirty = true;
    // the tile-ordered node record (Tiling::sx/sy/sz): 0 = stale, 1 = FP64 positions,
    // 2 = displacements x - X0 (FP32 mode); stale again whenever the positions change
    int stage_content = 0;
    // set once a caller has taken the positions' device pointers: it may write them at
    // any time, so the derived records are rebuilt before every evaluation
    bool positions_exposed = false;
    int* d_conn = nullptr;
    double* f_int = nullptr;
    double* f_ext = nullptr;
    float* f_int32 = nullptr;
    bool f_int_from32 = false;  // last fused evaluation wrote f_int32
    double* detJ = nullptr;     // reference layout E*nqp
    double* Pst = nullptr;      // reference layout E*nqp*9 (lazy)

    tlfea::Tiling tl;

    // node -> (element, slot) incidence in element order (cpu_utils.cc:97-109)
    int* inc_off = nullptr;
    int* inc_e = nullptr;
    int* inc_a = nullptr;
    std::vector<int> h_inc_off, h_inc_e, h_inc_a;

    // node-level pattern, shared by the mass CSR and the 3x3-block stiffness
    std::vector<int> h_pat_off, h_pat_col;
    int* pat_off = nullptr;
    int* pat_col = nullptr;
    long long pat_nnz = 0;
    double* m_val = nullptr;

    int n_constraint = 0;
    std::vector<int> h_fixed;
    int* fixed = nullptr;
    double* c = nullptr;
    int *jt_off = nullptr, *jt_col = nullptr;
    double* jt_val = nullptr;
    int *j_off = nullptr, *j_col = nullptr;
    double* j_val = nullptr;

    // error word set by kernels whose bounded waits ran out (checked at sync points)
    int* d_err = nullptr;
    // grid of the persistent force pipeline per (FP32?, damping?), 0 = not yet sized
    int pipe_grid[4] = {0, 0, 0, 0};
    // launch configuration (tlfea_element_set_launch_config): force kernel
    // 0 = TMA pipeline, 1 = one tile per block; cap on the pipeline grid (0 = none)
    int force_kernel = 0;
    int pipe_grid_limit = 0;
};

// The positions changed: the records derived from them (FP32 mode's displacement u64,
// the tile-ordered node record) are rebuilt before the next force evaluation.
inline void positions_changed(tlfea_element_s* h) {
    h->u_dirty = true;
    h->stage_content = 0;
}

namespace tlfea {
// Implemented in element.cu, used by the solvers.
int element_build_pattern(tlfea_element_s* h);
int element_force(tlfea_element_s* h, const double* d_v, bool fp32);
int element_refresh_u64(tlfea_element_s* h);
// Rebuild the tile-ordered node record (FP64 positions, or FP32 mode displacements) if stale.
int element_refresh_record(tlfea_element_s* h, bool fp32);

// Barycentric coordinates of the element's quadrature points.
inline QpBary qp_bary(const tlfea_element_s* h) {
    QpBary b;
    for (int q = 0; q < 5; ++q) {
        b.L[q][0] = 1.0 - h->qx[q] - h->qy[q] - h->qz[q];
        b.L[q][1] = h->qx[q];
        b.L[q][2] = h->qy[q];
        b.L[q][3] = h->qz[q];
    }
    return b;
}
}  // namespace tlfea
