// SIMPLE-pass assembly kernels for sm_100a (FP64).  Built with -fmad=false:
// every expression below is evaluated as the plain IEEE sequence the
// reference's C++ spells out (FlowSolver.inl), so the assembled coefficients
// equal the CPU oracle's bit for bit.
//
// Design: cell-centric gathers.  One thread owns one cell and walks its six
// faces in reference face order (sface), recomputing the face quantity it
// needs from face geometry and the two adjacent cells.  Every accumulation a
// reference face loop scatters into a cell happens here inside that cell's
// thread in the same order, so there are no atomics and results are
// deterministic.  Face-owned outputs (mass flux) come from face-parallel
// kernels.  All kernels are HBM-bandwidth bound.
#include "flow_kernels.cuh"
#include "mc_reduce.cuh"

namespace mcb {

namespace {

__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }  // std::max

// solve (FlowSolver.inl:895-915): Cramer's rule on the symmetric LSQ matrix.
__device__ __forceinline__ void cramer(double A00, double A10, double A20, double A11, double A21, double A22,
                                       const double b0, const double b1, const double b2, double &o0, double &o1,
                                       double &o2)
{
    const double A01 = A10, A02 = A20, A12 = A21;
    const double det = (A00 * (A11 * A22 - A21 * A12)) - (A01 * (A10 * A22 - A20 * A12)) +
                       (A02 * (A10 * A21 - A20 * A11));
    double invdet = 0.0;
    if (det != 0.0) invdet = 1 / det;
    o0 = (b0 * invdet * (A11 * A22 - A21 * A12)) + (b1 * invdet * (A21 * A02 - A01 * A22)) +
         (b2 * invdet * (A01 * A12 - A11 * A02));
    o1 = (b0 * invdet * (A12 * A20 - A10 * A22)) + (b1 * invdet * (A00 * A22 - A20 * A02)) +
         (b2 * invdet * (A10 * A02 - A00 * A12));
    o2 = (b0 * invdet * (A10 * A21 - A20 * A11)) + (b1 * invdet * (A20 * A01 - A00 * A21)) +
         (b2 * invdet * (A00 * A11 - A10 * A01));
}

__device__ __forceinline__ int grid_stride_start() { return blockIdx.x * blockDim.x + threadIdx.x; }

// The FP32 copy of an assembled row for the refined solves, written by the
// assembly kernel itself: the row, scaled by 1 / diag (1 when diag is 0) when
// f.scale_rows is set, with its six values stored by direction (slot k of
// code word cw holds direction (cw >> 3k) & 7, or 7 for an unused slot), or
// in slot order without codes -- the same values the separate rounding
// passes (k_round_ell, k_amg_round_level0) write.
__device__ __forceinline__ void store_fp32_row(const Fp32Rows &f, int N, int c, double diag, const double (&offv)[6])
{
    const double sc = f.scale_rows ? (diag != 0.0 ? 1.0 / diag : 1.0) : 1.0;
    f.d32[c] = (float)(diag * sc);
    if (!f.code) {
#pragma unroll
        for (int k = 0; k < 6; k++) f.o32[(size_t)k * N + c] = (float)(offv[k] * sc);
        return;
    }
    const uint32_t cw = f.code[c];
    float o[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const unsigned d = (cw >> (3 * k)) & 7u;
        const float v = (float)(offv[k] * sc);
#pragma unroll
        for (int q = 0; q < 6; q++) o[q] = (d == (unsigned)q) ? v : o[q];
    }
#pragma unroll
    for (int q = 0; q < 6; q++) f.o32[(size_t)q * N + c] = o[q];
}

// Row c stored by direction into out (see k_dir_rows64).
// Off-diagonal values of row c as RowStore says.
__device__ __forceinline__ void store_row(const RowStore &rs, double *out, int N, int c, const double (&offv)[6])
{
    if (!rs.code) {
#pragma unroll
        for (int k = 0; k < 6; k++) out[(size_t)k * N + c] = offv[k];
        return;
    }
    const uint32_t cw = rs.code[c];
    double o[6];
#pragma unroll
    for (int q = 0; q < 6; q++) o[q] = 0.0;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const unsigned d = (cw >> (3 * k)) & 7u;
        const unsigned p = d < 6 ? (rs.pos >> (3 * d)) & 7u : 7u;
#pragma unroll
        for (int q = 0; q < 6; q++) o[q] = (p == (unsigned)q) ? offv[k] : o[q];
    }
#pragma unroll
    for (int q = 0; q < 6; q++) out[(size_t)q * N + c] = o[q];
}

__device__ __forceinline__ void store_dir_row(const uint32_t cw, const double (&offv)[6], double *out, int N, int c,
                                              int sym)
{
    double o[6];
#pragma unroll
    for (int d = 0; d < 6; d++) o[d] = 0.0;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const unsigned d = (cw >> (3 * k)) & 7u;
#pragma unroll
        for (int q = 0; q < 6; q++) o[q] = (d == (unsigned)q) ? offv[k] : o[q];
    }
    if (sym) {
#pragma unroll
        for (int j = 0; j < 3; j++) out[(size_t)j * N + c] = o[2 * j + 1];
    } else {
#pragma unroll
        for (int q = 0; q < 6; q++) out[(size_t)q * N + c] = o[q];
    }
}

} // namespace

// ------------------------------------------------------------- gradients
// get_phi_gradients / get_phi_gradient (FlowSolver.inl:738-803, 917-1063).
// Over slot f in cell_faces order: dX = x_nbr - x_c (equal to the reference's
// mask * (x1 - x0)), boundary dX = x_face - x_c; dphi likewise, or 0 on
// boundary faces for pressure-like fields.
// The five-field form is held to 3 blocks of 256 per SM (80 registers, a few
// spilled) instead of the 106 registers and 2 blocks it takes unbounded.
template <int NF>
__device__ __forceinline__ void lsq_cell(int N, const int *__restrict__ nbr, const int *__restrict__ fc1,
                                         const double *__restrict__ xc, const double *__restrict__ yc,
                                         const double *__restrict__ zc, const double *__restrict__ xf,
                                         const double *__restrict__ yf, const double *__restrict__ zf,
                                         const GradArgs<NF> &a, int c)
{
    const double x = xc[c], y = yc[c], z = zc[c];
    double pc[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) pc[k] = a.phi[k][c];
    double A00 = 0.0, A10 = 0.0, A20 = 0.0, A11 = 0.0, A21 = 0.0, A22 = 0.0;
    double b[NF][3];
#pragma unroll
    for (int k = 0; k < NF; k++) b[k][0] = b[k][1] = b[k][2] = 0.0;
#pragma unroll
    for (int f = 0; f < 6; f++) {
        const int n = nbr[(size_t)f * N + c];
        double dx, dy, dz, dphi[NF];
        if (n >= 0) {
            dx = xc[n] - x;
            dy = yc[n] - y;
            dz = zc[n] - z;
#pragma unroll
            for (int k = 0; k < NF; k++) dphi[k] = a.phi[k][n] - pc[k];
        } else {
            const int face = -1 - n;
            dx = xf[face] - x;
            dy = yf[face] - y;
            dz = zf[face] - z;
            const int slot = fc1[face];
#pragma unroll
            for (int k = 0; k < NF; k++) dphi[k] = ((a.zero_boundary >> k) & 1) ? 0.0 : a.phi[k][slot] - pc[k];
        }
        A00 += (dx * dx);
        A10 += (dx * dy);
        A20 += (dx * dz);
        A11 += (dy * dy);
        A21 += (dy * dz);
        A22 += (dz * dz);
#pragma unroll
        for (int k = 0; k < NF; k++) {
            b[k][0] += (dx * dphi[k]);
            b[k][1] += (dy * dphi[k]);
            b[k][2] += (dz * dphi[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < NF; k++) {
        double gx, gy, gz;
        cramer(A00, A10, A20, A11, A21, A22, b[k][0], b[k][1], b[k][2], gx, gy, gz);
        a.gx[k][c] = gx;
        a.gy[k][c] = gy;
        a.gz[k][c] = gz;
    }
}

template <int NF>
__global__ void __launch_bounds__(MCB_THREADS, NF > 1 ? 3 : 0) k_lsq_gradients(int N, const int *__restrict__ nbr,
                                                              const int *__restrict__ fc1, const double *__restrict__ xc,
                                                              const double *__restrict__ yc,
                                                              const double *__restrict__ zc,
                                                              const double *__restrict__ xf,
                                                              const double *__restrict__ yf,
                                                              const double *__restrict__ zf, GradArgs<NF> a)
{
    const int c = grid_stride_start();
    if (c < N) lsq_cell<NF>(N, nbr, fc1, xc, yc, zc, xf, yf, zf, a, c);
}

void launch_lsq_gradients5(cudaStream_t s, int N, const int *nbr, const int *fc1, const double *xc,
                           const double *yc, const double *zc, const double *xf, const double *yf, const double *zf,
                           const GradArgs<5> &a)
{
    k_lsq_gradients<5><<<(N + MCB_THREADS - 1) / MCB_THREADS, MCB_THREADS, 0, s>>>(N, nbr, fc1, xc, yc, zc, xf, yf,
                                                                                  zf, a);
}

void launch_lsq_gradients1(cudaStream_t s, int N, const int *nbr, const int *fc1, const double *xc,
                           const double *yc, const double *zc, const double *xf, const double *yf, const double *zf,
                           const GradArgs<1> &a)
{
    k_lsq_gradients<1><<<(N + MCB_THREADS - 1) / MCB_THREADS, MCB_THREADS, 0, s>>>(N, nbr, fc1, xc, yc, zc, xf, yf,
                                                                                  zf, a);
}

void launch_lsq_gradients6(cudaStream_t s, int N, const int *nbr, const int *fc1, const double *xc,
                           const double *yc, const double *zc, const double *xf, const double *yf, const double *zf,
                           const GradArgs<6> &a)
{
    k_lsq_gradients<6><<<(N + MCB_THREADS - 1) / MCB_THREADS, MCB_THREADS, 0, s>>>(N, nbr, fc1, xc, yc, zc, xf, yf,
                                                                                  zf, a);
}

// -------------------------------------------------------------- precomp_AU
// precomp_AU (FlowSolver.inl:1065-1104): inlet/outlet viscous part plus rho V / dt.
__global__ void __launch_bounds__(MCB_THREADS) k_precomp_au(Physics ph, MeshArgs m, const double *__restrict__ mdot,
                                                            double *__restrict__ AU)
{
    const int N = ph.N;
    const int c = grid_stride_start();
    if (c >= N) return;
    double a = 0.0;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const int face = m.sface[(size_t)k * N + c];
        const int c1 = m.fc1[face];
        if (c1 < N) continue;
        const int t = ph.btype[c1 - N];
        if (t == INLET || t == OUTLET) {
            const double VisFace = ph.mu * m.rl[face];
            const double f = -VisFace + smin(mdot[face], 0.0);
            a = a - f;
        }
    }
    const double f = m.rho[c] * m.vol[c] * ph.rdelta;
    a += f;
    AU[c] = a;
}

// ---------------------------------------------------------------- momentum
// calculate_flux_UVW (FlowSolver.inl:1377-1653), the cell source terms of
// calculate_UVW (:1689-1729) and setup/update_sparse_matrix (:1186-1339) for
// the three velocity components at once.  The U, V and W systems share the
// off-diagonal coefficients and, bit for bit, the diagonal.
__global__ void __launch_bounds__(MCB_THREADS, 4) k_momentum_assemble(Physics ph, MeshArgs m, MomentumArgs a)
{
    const int N = ph.N;
    const int c = grid_stride_start();
    if (c >= N) return;
    const double xcc = m.xc[c], ycc = m.yc[c], zcc = m.zc[c];
    const double Uc = a.U[c], Vc = a.V[c], Wc = a.W[c];
    const unsigned own = m.own[c];
    double su = 0.0, sv = 0.0, sw = 0.0, ac = 0.0;
    double offv[6];
    unsigned internal = 0u;
    const double mu = ph.mu;
    for (int k = 0; k < 6; k++) {
        const int face = m.sface[(size_t)k * N + c];
        const int nb = m.col[(size_t)k * N + c];
        const double Sx = m.Sx[face], Sy = m.Sy[face], Sz = m.Sz[face];
        if (nb != c) {
            const bool c_is_c0 = (own >> k) & 1u;
            const int c0 = c_is_c0 ? c : nb, c1 = c_is_c0 ? nb : c;
            internal |= 1u << k;
            const double l0 = m.lam[face];
            const double l1 = 1.0 - l0;
            double g0[9], g1[9], x0[3], x1[3];  // values at c0 and c1
#pragma unroll
            for (int d = 0; d < 3; d++) {
                g0[d] = a.gU[d][c0];
                g1[d] = a.gU[d][c1];
                g0[3 + d] = a.gV[d][c0];
                g1[3 + d] = a.gV[d][c1];
                g0[6 + d] = a.gW[d][c0];
                g1[6 + d] = a.gW[d][c1];
            }
            x0[0] = m.xc[c0];
            x0[1] = m.yc[c0];
            x0[2] = m.zc[c0];
            x1[0] = m.xc[c1];
            x1[1] = m.yc[c1];
            x1[2] = m.zc[c1];
            const double dUx = g0[0] * l0 + g1[0] * l1;
            const double dUy = g0[1] * l0 + g1[1] * l1;
            const double dUz = g0[2] * l0 + g1[2] * l1;
            const double dVx = g0[3] * l0 + g1[3] * l1;
            const double dVy = g0[4] * l0 + g1[4] * l1;
            const double dVz = g0[5] * l0 + g1[5] * l1;
            const double dWx = g0[6] * l0 + g1[6] * l1;
            const double dWy = g0[7] * l0 + g1[7] * l1;
            const double dWz = g0[8] * l0 + g1[8] * l1;
            const double Visac = mu * l0 + mu * l1;
            const double VisFace = Visac * m.rl[face];
            const double Xx = x1[0] - x0[0], Xy = x1[1] - x0[1], Xz = x1[2] - x0[2];
            const double md = a.mdot[face];
            const double fude = Visac * ((dUx + dUx) * Sx + (dUy + dVx) * Sy + (dUz + dWx) * Sz);
            const double fvde = Visac * ((dUy + dVx) * Sx + (dVy + dVy) * Sy + (dVz + dWy) * Sz);
            const double fwde = Visac * ((dUz + dWx) * Sx + (dWy + dVz) * Sy + (dWz + dWz) * Sz);
            const double fudi = VisFace * (dUx * Xx + dUy * Xy + dUz * Xz);
            const double fvdi = VisFace * (dVx * Xx + dVy * Xy + dVz * Xz);
            const double fwdi = VisFace * (dWx * Xx + dWy * Xy + dWz * Xz);
            // The deferred-correction blend is GammaBlend = 0 (:1387) and is omitted.
            if (c == c0) {
                su = su + fude - fudi;
                sv = sv + fvde - fvdi;
                sw = sw + fwde - fwdi;
                offv[k] = -VisFace + smin(md, 0.0);  // face_fields.cell1, column c1
            } else {
                su = su - fude + fudi;
                sv = sv - fvde + fvdi;
                sw = sw - fwde + fwdi;
                offv[k] = -VisFace - smax(md, 0.0);  // face_fields.cell0, column c0
            }
        } else {
            offv[k] = 0.0;
            const int c1 = m.fc1[face];
            const int side = c1 - N;
            const int t = ph.btype[side];
            const double Xx = m.xf[face] - xcc, Xy = m.yf[face] - ycc, Xz = m.zf[face] - zcc;
            if (t == INLET || t == OUTLET) {
                const double dUx = a.gU[0][c], dUy = a.gU[1][c], dUz = a.gU[2][c];
                const double dVx = a.gV[0][c], dVy = a.gV[1][c], dVz = a.gV[2][c];
                const double dWx = a.gW[0][c], dWy = a.gW[1][c], dWz = a.gW[2][c];
                double UF, VF, WF, Visac;
                if (t == INLET) {
                    UF = ph.u_in;
                    VF = 0.0;
                    WF = 0.0;
                    Visac = ph.inlet_mu;
                } else {
                    UF = Uc;
                    VF = Vc;
                    WF = Wc;
                    Visac = mu;
                }
                const double VisFace = Visac * m.rl[face];
                const double fude = Visac * ((dUx + dUx) * Sx + (dUy + dVx) * Sy + (dUz + dWx) * Sz);
                const double fvde = Visac * ((dUy + dVx) * Sx + (dVy + dVy) * Sy + (dVz + dWy) * Sz);
                const double fwde = Visac * ((dUz + dWx) * Sx + (dWy + dVz) * Sy + (dWz + dWz) * Sz);
                const double fudi = VisFace * (dUx * Xx + dUy * Xy + dUz * Xz);
                const double fvdi = VisFace * (dVx * Xx + dVy * Xy + dVz * Xz);
                const double fwdi = VisFace * (dWx * Xx + dWy * Xy + dWz * Xz);
                double md = a.mdot[face];
                if (t == OUTLET && md < 0.0) {  // :1576-1580
                    md = 1e-15;
                    a.mdot[face] = md;
                }
                const double f = -VisFace + smin(md, 0.0);
                ac = ac - f;
                su = su - f * UF + fude - fudi;
                sv = sv - f * VF + fvde - fvdi;
                sw = sw - f * WF + fwde - fwdi;
                if (face == ph.last_bface[side]) {
                    a.U[c1] = UF;
                    a.V[c1] = VF;
                    a.W[c1] = WF;
                }
            } else if (t == WALL) {
                const double Visac = mu;
                const double coef = Visac * m.rl[face];
                const double Upx = Uc - 0., Upy = Vc - 0., Upz = Wc - 0.;
                const double smag = sqrt(Sx * Sx + Sy * Sy + Sz * Sz);
                const double nx = Sx / smag, ny = Sy / smag, nz = Sz / smag;
                const double dp = Upx * nx + Upy * ny + Upz * nz;
                const double Utx = Upx - nx * dp, Uty = Upy - ny * dp, Utz = Upz - nz * dp;
                const double Uvel = fabs(Utx) + fabs(Uty) + fabs(Utz);
                double fx = 0.0, fy = 0.0, fz = 0.0;
                if (Uvel > 0.0) {
                    const double dist = sqrt(Xx * Xx + Xy * Xy + Xz * Xz);
                    const double s = m.area[face] * Visac;
                    fx = Utx * s / dist;
                    fy = Uty * s / dist;
                    fz = Utz * s / dist;
                }
                ac = ac + coef;
                su = su + coef * Uc - fx;
                sv = sv + coef * Vc - fy;
                sw = sw + coef * Wc - fz;
                if (face == ph.last_bface[side]) {
                    a.U[c1] = 0.;
                    a.V[c1] = 0.;
                    a.W[c1] = 0.;
                }
            }
        }
    }
    const double vol = m.vol[c], rho = m.rho[c];
    const double BodyForce = -0.001 * rho * vol * (a.T[c] - ph.T_ref);  // :1689-1697
    su += 0.0 * BodyForce;
    sv += -9.81 * BodyForce;
    sw += 0.0 * BodyForce;
    su -= a.gP[0][c] * vol;  // :1700-1705
    sv -= a.gP[1][c] * vol;
    sw -= a.gP[2][c] * vol;
    const double f = rho * vol * ph.rdelta;  // :1708-1721
    su += f * Uc;
    sv += f * Vc;
    sw += f * Wc;
    ac += f;
    if (ph.mode == 1 && a.src) {  // particle momentum (left commented out at :1723-1729)
        su += a.src[c];
        sv += a.src[(size_t)N + c];
        sw += a.src[2 * (size_t)N + c];
    }
    for (int k = 0; k < 6; k++)  // setup_sparse_matrix diagonal, :1242-1243
        if ((internal >> k) & 1u) ac -= offv[k];
    const double URF = ph.urf_u;
    const double RURF = 1. / URF;
    ac *= RURF;
    a.b[c] = su + (1.0 - URF) * ac * Uc;
    a.b[(size_t)N + c] = sv + (1.0 - URF) * ac * Vc;
    a.b[2 * (size_t)N + c] = sw + (1.0 - URF) * ac * Wc;
    a.AU[c] = ac;
    store_row(a.store, a.off, N, c, offv);
    if (a.f32.d32) store_fp32_row(a.f32, N, c, ac, offv);
}


// ------------------------------------------------------------- temperature
// FluxScalar(TEMP) (FlowSolver.inl:2516-2744), unsteady term and
// setup_sparse_matrix of Scalar_solve (:2885-2953).
// One cell's row; returns |div(mdot) - mass source| of the cell (the mass
// imbalance after the pass: the temperature stage reads the pass's final
// face fluxes anyway).
__device__ __forceinline__ double temperature_row(const Physics &ph, const MeshArgs &m, const ScalarArgs &a, int c)
{
    const int N = ph.N;
    double div = 0.0;
    const double xcc = m.xc[c], ycc = m.yc[c], zcc = m.zc[c];
    const double Tc = a.phi[c];
    const double mu = ph.mu;
    double st = 0.0, at = 0.0, offv[6];
    unsigned internal = 0u;
    for (int k = 0; k < 6; k++) {
        const int face = m.sface[(size_t)k * N + c];
        const int c0 = m.fc0[face], c1 = m.fc1[face];
        const double Sx = m.Sx[face], Sy = m.Sy[face], Sz = m.Sz[face];
        const double md = a.mdot[face];
        div += (c0 == c) ? md : -md;
        if (c1 < N) {
            internal |= 1u << k;
            const double l0 = m.lam[face];
            const double l1 = 1.0 - l0;
            double Visac = mu * l0 + mu * l1;
            Visac -= mu;
            Visac = (mu + Visac / 0.9) / 0.6905;
            // the gradient and centre at c0 and at c1, all loaded before use
            double g0[3], g1[3], x0[3], x1[3];
#pragma unroll
            for (int q = 0; q < 3; q++) {
                g0[q] = a.g[q][c0];
                g1[q] = a.g[q][c1];
            }
            x0[0] = m.xc[c0];
            x0[1] = m.yc[c0];
            x0[2] = m.zc[c0];
            x1[0] = m.xc[c1];
            x1[1] = m.yc[c1];
            x1[2] = m.zc[c1];
            const double dx = g0[0] * l0 + g1[0] * l1;
            const double dy = g0[1] * l0 + g1[1] * l1;
            const double dz = g0[2] * l0 + g1[2] * l1;
            const double Xx = x1[0] - x0[0], Xy = x1[1] - x0[1], Xz = x1[2] - x0[2];
            const double VisFace = Visac * m.rl[face];
            const double fde1 = Visac * (dx * Sx + dy * Sy + dz * Sz);
            const double fdi = VisFace * (dx * Xx + dy * Xy + dz * Xz);
            if (c == c0) {
                st = st + fde1 - fdi;
                offv[k] = -VisFace + smin(md, 0.0);
            } else {
                st = st - fde1 + fdi;
                offv[k] = -VisFace - smax(md, 0.0);
            }
        } else {
            offv[k] = 0.0;
            const int side = c1 - N;
            const int t = ph.btype[side];
            const double dx = a.g[0][c], dy = a.g[1][c], dz = a.g[2][c];
            const double Xx = m.xf[face] - xcc, Xy = m.yf[face] - ycc, Xz = m.zf[face] - zcc;
            if (t == INLET) {
                const double PhiFace = ph.T_ref;
                double Visac = ph.inlet_mu;
                Visac -= mu;
                Visac = (mu + Visac / 0.9) / 0.6905;
                const double VisFace = Visac * m.rl[face];
                const double fde = Visac * (dx * Sx + dy * Sy + dz * Sz);
                const double fdi = VisFace * (dx * Xx + dy * Xy + dz * Xz);
                const double f = -VisFace + smin(md, 0.0);
                at = at - f;
                st = st - f * PhiFace + fde - fdi;
                if (face == ph.last_bface[side]) a.phi[c1] = PhiFace;
            } else if (t == OUTLET) {
                double Visac = mu;
                Visac -= mu;
                Visac = (mu + Visac / 0.9) / 0.6905;
                const double PhiFace = Tc + (dx * Xx + dy * Xy + dz * Xz);
                const double VisFace = Visac * m.rl[face];
                const double fde = Visac * (dx * Sx + dy * Sy + dz * Sz);
                const double fdi = VisFace * (dx * Xx + dy * Xy + dz * Xz);
                st = st + fde - fdi;
                if (face == ph.last_bface[side]) a.phi[c1] = PhiFace;
            } else if (t == WALL) {
                if (face == ph.last_bface[side]) a.phi[c1] = Tc;
            }
        }
    }
    const double f = m.rho[c] * m.vol[c] * ph.rdelta;
    st += f * Tc;
    at += f;
    if (ph.mode == 1 && a.src) st += a.src[3 * (size_t)N + c];  // particle energy (commented out at :2919-2925)
    for (int k = 0; k < 6; k++)
        if ((internal >> k) & 1u) at -= offv[k];
    const double URF = ph.urf_T;
    const double RURF = 1. / URF;
    at *= RURF;
    a.b[c] = st + (1.0 - URF) * at * Tc;
    a.diag[c] = at;
    store_row(a.store, a.off, N, c, offv);
    if (a.f32.d32) store_fp32_row(a.f32, N, c, at, offv);
    if (ph.mode == 1 && a.src) div -= a.src[4 * (size_t)N + c];
    return fabs(div);
}

// The imbalance maximum: a warp maximum, then one atomicMax per warp on the
// bits of the (non-negative) value -- for non-negative doubles the order of
// the bit patterns is the order of the values, and a maximum does not depend
// on the order of the updates.  *imbalance must be zero before the launch.
__global__ void __launch_bounds__(MCB_THREADS, 4) k_temperature_assemble(Physics ph, MeshArgs m, ScalarArgs a)
{
    const int c = grid_stride_start();
    double v = 0.0;
    if (c < ph.N) v = temperature_row(ph, m, a, c);
    if (a.imbalance) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
        if ((threadIdx.x & 31) == 0 && v > 0.0)
            atomicMax((unsigned long long *)a.imbalance, (unsigned long long)__double_as_longlong(v));
    }
}

// ------------------------------------------------------ other scalar transports
// Scalar_solve (FlowSolver.inl:2885-2955) for TE, ED, FUL, PRO, VARF, VARP:
// FluxScalar (:2516-2744) with the scalar's diffusivity and inlet value, the
// unsteady term, for TE and ED the k-epsilon sources and wall functions of
// solveTurbulenceModels (:2746-2883), then setup_sparse_matrix (:1186-1297)
// with under-relaxation 0.5 (TE, ED) or 0.95.  One thread per cell as in the
// temperature kernel: the cell's faces in reference face order, then its
// wall faces again in that order for the wall functions.

namespace {

// Effective diffusivity from Visac = face viscosity - mu (FluxScalar,
// FlowSolver.inl:2543-2561).
template <int TYPE>
__device__ __forceinline__ double scalar_visac(double mu, double v)
{
    if (TYPE == SC_TERBTE) return mu + v;
    if (TYPE == SC_TERBED) return mu + v / 1.219;
    return (mu + v / 0.9) / 0.9;
}

// x^1.5 rounded once: s = sqrt(x) is corrected by the exact residual
// x - s^2 (one Newton step on the square root), and x * s is formed exactly
// as a sum of two doubles (the FMA product split of Ogita, Rump and Oishi,
// "Accurate sum and dot product", SIAM J. Sci. Comput. 2005), so the result
// carries about 100 bits before its single rounding.
__device__ __forceinline__ double pow_three_halves(double x)
{
    const double s = sqrt(x);
    const double e = fma(-s, s, x);
    const double c = e / (2.0 * s);
    const double p = x * s;
    const double pl = fma(x, s, -p);
    return p + (pl + x * c);
}

} // namespace

template <int TYPE>
__global__ void __launch_bounds__(MCB_THREADS, 4) k_scalar_assemble(Physics ph, MeshArgs m, ScalarArgs a, TurbArgs t)
{
    const int N = ph.N;
    const int c = grid_stride_start();
    if (c >= N) return;
    const double xcc = m.xc[c], ycc = m.yc[c], zcc = m.zc[c];
    double phic = a.phi[c];
    const double mu = ph.mu;
    double st = 0.0, at = 0.0, offv[6];
    unsigned internal = 0u, wall = 0u;
    for (int k = 0; k < 6; k++) {
        const int face = m.sface[(size_t)k * N + c];
        const int c0 = m.fc0[face], c1 = m.fc1[face];
        const double Sx = m.Sx[face], Sy = m.Sy[face], Sz = m.Sz[face];
        const double md = a.mdot[face];
        if (c1 < N) {
            internal |= 1u << k;
            const double l0 = m.lam[face];
            const double l1 = 1.0 - l0;
            double Visac = mu * l0 + mu * l1;
            Visac -= mu;
            Visac = scalar_visac<TYPE>(mu, Visac);
            const double dx = a.g[0][c0] * l0 + a.g[0][c1] * l1;
            const double dy = a.g[1][c0] * l0 + a.g[1][c1] * l1;
            const double dz = a.g[2][c0] * l0 + a.g[2][c1] * l1;
            const double Xx = m.xc[c1] - m.xc[c0], Xy = m.yc[c1] - m.yc[c0], Xz = m.zc[c1] - m.zc[c0];
            const double VisFace = Visac * m.rl[face];
            const double fde1 = Visac * (dx * Sx + dy * Sy + dz * Sz);
            const double fdi = VisFace * (dx * Xx + dy * Xy + dz * Xz);
            if (c == c0) {
                st = st + fde1 - fdi;
                offv[k] = -VisFace + smin(md, 0.0);
            } else {
                st = st - fde1 + fdi;
                offv[k] = -VisFace - smax(md, 0.0);
            }
        } else {
            offv[k] = 0.0;
            const int side = c1 - N;
            const int bt = ph.btype[side];
            const double dx = a.g[0][c], dy = a.g[1][c], dz = a.g[2][c];
            const double Xx = m.xf[face] - xcc, Xy = m.yf[face] - ycc, Xz = m.zf[face] - zcc;
            if (bt == INLET) {
                const double PhiFace = ph.sc_inlet[TYPE];
                double Visac = ph.inlet_mu;
                Visac -= mu;
                Visac = scalar_visac<TYPE>(mu, Visac);
                const double VisFace = Visac * m.rl[face];
                const double fde = Visac * (dx * Sx + dy * Sy + dz * Sz);
                const double fdi = VisFace * (dx * Xx + dy * Xy + dz * Xz);
                const double f = -VisFace + smin(md, 0.0);
                at = at - f;
                st = st - f * PhiFace + fde - fdi;
                if (face == ph.last_bface[side]) a.phi[c1] = PhiFace;
            } else if (bt == OUTLET) {
                double Visac = mu;
                Visac -= mu;
                Visac = scalar_visac<TYPE>(mu, Visac);
                const double PhiFace = phic + (dx * Xx + dy * Xy + dz * Xz);
                const double VisFace = Visac * m.rl[face];
                const double fde = Visac * (dx * Sx + dy * Sy + dz * Sz);
                const double fdi = VisFace * (dx * Xx + dy * Xy + dz * Xz);
                st = st + fde - fdi;
                if (face == ph.last_bface[side]) a.phi[c1] = PhiFace;
            } else if (bt == WALL) {
                wall |= 1u << k;
                if (face == ph.last_bface[side]) a.phi[c1] = phic;
            }
        }
    }
    const double rho = m.rho[c], vol = m.vol[c];
    const double f = rho * vol * ph.rdelta;
    st += f * phic;
    at += f;
    if (TYPE == SC_TERBTE) {
        // production (zero: the turbulent viscosity is mu - mu) and
        // dissipation, :2754-2775
        const double uxx = t.gU[0][c], uxy = t.gU[1][c], uxz = t.gU[2][c];
        const double vxx = t.gV[0][c], vxy = t.gV[1][c], vxz = t.gV[2][c];
        const double wxx = t.gW[0][c], wxy = t.gW[1][c], wxz = t.gW[2][c];
        const double s1 = (uxx + uxx) * uxx + (uxy + vxx) * uxy + (uxz + wxx) * uxz;
        const double s2 = (vxx + uxy) * vxx + (vxy + vxy) * vxy + (vxz + wxy) * vxz;
        const double s3 = (wxx + uxz) * wxx + (wxy + vxz) * wxy + (wxz + wxz) * wxz;
        const double VisT = mu - mu;
        double TP = VisT * (s1 + s2 + s3);
        const double Dis = rho * t.ED[c];
        st = st + TP * vol;
        at = at + Dis / (phic + 0.000000000000000001) * vol;
        // wall functions, :2778-2822
        for (int k = 0; k < 6; k++) {
            if (!((wall >> k) & 1u)) continue;
            const int face = m.sface[(size_t)k * N + c];
            st = st - TP * vol;
            const double Xx = m.xf[face] - xcc, Xy = m.yf[face] - ycc, Xz = m.zf[face] - zcc;
            const double Upx = t.U[c] - 0., Upy = t.V[c] - 0., Upz = t.W[c] - 0.;
            const double Sx = m.Sx[face], Sy = m.Sy[face], Sz = m.Sz[face];
            const double mag = sqrt(Sx * Sx + Sy * Sy + Sz * Sz);
            const double nx = Sx / mag, ny = Sy / mag, nz = Sz / mag;
            const double dp = Upx * nx + Upy * ny + Upz * nz;
            const double Utx = Upx - nx * dp, Uty = Upy - ny * dp, Utz = Upz - nz * dp;
            const double Uvel = sqrt(Utx * Utx + Uty * Uty + Utz * Utz);
            const double distance_to_face = sqrt(Xx * Xx + Xy * Xy + Xz * Xz);
            const double rkapdn = 1.0 / (0.419 * distance_to_face);
            const double Tau_w = mu * Uvel / distance_to_face;
            const double Utau = sqrt(Tau_w / rho);
            TP = Tau_w * Utau * rkapdn;
            st = st + TP * vol;
            const double DisP = ph.cmu75 * sqrt(phic) * rkapdn;
            at = at + rho * DisP * vol;
        }
        t.TP[c] = TP;
    } else if (TYPE == SC_TERBED) {
        // epsilon sources, :2826-2831
        const double fact = phic / (t.TE[c] + 0.000000000000000001) * vol;
        st = st + 1.44 * fact * t.TP[c];
        at = at + 1.92 * fact * rho;
        if (wall) {
            // fixed dissipation at wall cells, their own side of face_fields
            // zeroed (:2835-2878): the row keeps only its diagonal
            const double turb = t.TE[c];
            double Dis = 0.0;
            for (int k = 0; k < 6; k++) {
                if (!((wall >> k) & 1u)) continue;
                const int face = m.sface[(size_t)k * N + c];
                const double Xx = m.xf[face] - xcc, Xy = m.yf[face] - ycc, Xz = m.zf[face] - zcc;
                const double distance = sqrt(Xx * Xx + Xy * Xy + Xz * Xz);
                Dis = ph.cmu75 * pow_three_halves(turb) / (distance * 0.419);
                const int side = m.fc1[face] - N;
                if (face == ph.last_bface[side]) a.phi[N + side] = Dis;
            }
            phic = Dis;
            st = Dis;
            at = 1;
            for (int k = 0; k < 6; k++) offv[k] = 0.0;
        }
    }
    for (int k = 0; k < 6; k++)
        if ((internal >> k) & 1u) at -= offv[k];
    const double URF = (TYPE == SC_TERBTE || TYPE == SC_TERBED) ? 0.5 : 0.95;
    const double RURF = 1. / URF;
    at *= RURF;
    a.b[c] = st + (1.0 - URF) * at * phic;
    a.diag[c] = at;
    store_row(a.store, a.off, N, c, offv);
}

void launch_scalar_assemble(cudaStream_t s, int type, const Physics &ph, const MeshArgs &m, const ScalarArgs &a,
                            const TurbArgs &t)
{
    const int grid = (ph.N + MCB_THREADS - 1) / MCB_THREADS;
    switch (type) {
    case SC_TERBTE: k_scalar_assemble<SC_TERBTE><<<grid, MCB_THREADS, 0, s>>>(ph, m, a, t); break;
    case SC_TERBED: k_scalar_assemble<SC_TERBED><<<grid, MCB_THREADS, 0, s>>>(ph, m, a, t); break;
    case SC_FUEL: k_scalar_assemble<SC_FUEL><<<grid, MCB_THREADS, 0, s>>>(ph, m, a, t); break;
    case SC_PROG: k_scalar_assemble<SC_PROG><<<grid, MCB_THREADS, 0, s>>>(ph, m, a, t); break;
    case SC_VARFU: k_scalar_assemble<SC_VARFU><<<grid, MCB_THREADS, 0, s>>>(ph, m, a, t); break;
    case SC_VARPR: k_scalar_assemble<SC_VARPR><<<grid, MCB_THREADS, 0, s>>>(ph, m, a, t); break;
    default: break;
    }
}

// Negative k or epsilon after the solve: list them (unordered, up to cap).
__global__ void __launch_bounds__(MCB_THREADS) k_scalar_negatives(int N, ClipArgs a)
{
    for (int c = grid_stride_start(); c < N; c += gridDim.x * blockDim.x) {
        if (a.phi[c] < 0.0) {
            const unsigned int i = atomicAdd(a.count, 1u);
            if (i < (unsigned int)a.cap) a.list[i] = c;
        }
    }
}

namespace {

// One cell of the reference's loop (FlowSolver.inl:2961-2983): the mean of
// its internal neighbours' current values, at least 1e-12.
__device__ void clip_cell(int N, const ClipArgs &a, int c)
{
    if (!(a.phi[c] < 0.0)) return;
    int count = 0;
    double phisum = 0.0;
    for (int j = 0; j < 6; j++) {
        const int nb = a.nbr[(size_t)j * N + c];
        if (nb >= 0) {
            count++;
            phisum += a.phi[nb];
        }
    }
    phisum = (phisum / count);
    a.phi[c] = smax(phisum, 0.000000000001);
}

} // namespace

// The listed cells, replaced one at a time in ascending caller order, so a
// cell sees the replaced values of the earlier cells and the old values of
// the later ones, as in the reference's sequential loop.  One block: the
// list (at most 4096 cells) is sorted in shared memory; a longer list falls
// back to one thread walking every cell in caller order.  Resets the count.
__global__ void __launch_bounds__(1024) k_scalar_clip(int N, ClipArgs a)
{
    constexpr int kCap = 4096;
    __shared__ int skey[kCap];
    __shared__ int sval[kCap];
    const unsigned int cnt = *a.count;
    if (cnt == 0) return;
    if (cnt > (unsigned int)a.cap || cnt > (unsigned int)kCap) {
        if (threadIdx.x == 0) {
            for (int o = 0; o < N; o++) clip_cell(N, a, a.o2n ? a.o2n[o] : o);
            *a.count = 0u;
        }
        return;
    }
    int n2 = 1;
    while (n2 < (int)cnt) n2 <<= 1;
    for (int i = threadIdx.x; i < n2; i += blockDim.x) {
        if (i < (int)cnt) {
            const int c = a.list[i];
            skey[i] = a.key ? a.key[c] : c;
            sval[i] = c;
        } else {
            skey[i] = 0x7fffffff;
            sval[i] = -1;
        }
    }
    __syncthreads();
    for (int k = 2; k <= n2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < n2; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    if ((skey[i] > skey[ixj]) == up) {
                        const int tk = skey[i], tv = sval[i];
                        skey[i] = skey[ixj];
                        sval[i] = sval[ixj];
                        skey[ixj] = tk;
                        sval[ixj] = tv;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < (int)cnt; i++) clip_cell(N, a, sval[i]);
        *a.count = 0u;
    }
}

// --------------------------------------------------------------- mass flux
// calculate_mass_flux face loop (FlowSolver.inl:1885-2007): Rhie-Chow flux
// and -ApV on internal faces; inlet, outlet and wall fluxes; partial sums
// of the boundary balance (:2010-2034), finished by the last block.
__global__ void __launch_bounds__(MCB_THREADS, 4) k_mass_flux(Physics ph, MeshArgs m, MassFluxArgs a)
{
    __shared__ double sh[3][MCB_THREADS];
    const int N = ph.N, F = m.F;
    double part[3] = {0.0, 0.0, 0.0};  // flow_in, flow_out, area_out
    for (int face = grid_stride_start(); face < F; face += gridDim.x * blockDim.x) {
        const int c0 = m.fc0[face], c1 = m.fc1[face];
        const double Sx = m.Sx[face], Sy = m.Sy[face], Sz = m.Sz[face];
        if (c1 < N) {
            const double l0 = m.lam[face];
            const double l1 = 1.0 - l0;
            const double dUx = a.gU[0][c0] * l0 + a.gU[0][c1] * l1;
            const double dUy = a.gU[1][c0] * l0 + a.gU[1][c1] * l1;
            const double dUz = a.gU[2][c0] * l0 + a.gU[2][c1] * l1;
            const double dVx = a.gV[0][c0] * l0 + a.gV[0][c1] * l1;
            const double dVy = a.gV[1][c0] * l0 + a.gV[1][c1] * l1;
            const double dVz = a.gV[2][c0] * l0 + a.gV[2][c1] * l1;
            const double dWx = a.gW[0][c0] * l0 + a.gW[0][c1] * l1;
            const double dWy = a.gW[1][c0] * l0 + a.gW[1][c1] * l1;
            const double dWz = a.gW[2][c0] * l0 + a.gW[2][c1] * l1;
            const double x0 = m.xc[c0], y0 = m.yc[c0], z0 = m.zc[c0];
            const double x1 = m.xc[c1], y1 = m.yc[c1], z1 = m.zc[c1];
            const double xf = m.xf[face], yf = m.yf[face], zf = m.zf[face];
            const double Xacx = x1 * l1 + x0 * l0, Xacy = y1 * l1 + y0 * l0, Xacz = z1 * l1 + z0 * l0;
            const double dlx = xf - Xacx, dly = yf - Xacy, dlz = zf - Xacz;
            const double UF = a.U[c1] * l1 + a.U[c0] * l0 + (dUx * dlx + dUy * dly + dUz * dlz);
            const double VF = a.V[c1] * l1 + a.V[c0] * l0 + (dVx * dlx + dVy * dly + dVz * dlz);
            const double WF = a.W[c1] * l1 + a.W[c0] * l0 + (dWx * dlx + dWy * dly + dWz * dlz);
            const double densityf = m.rho[c0] * l0 + m.rho[c1] * l1;
            double md = densityf * (UF * Sx + VF * Sy + WF * Sz);
            const double smag = sqrt(Sx * Sx + Sy * Sy + Sz * Sz);
            const double nx = Sx / smag, ny = Sy / smag, nz = Sz / smag;
            const double d0 = (xf - x0) * nx + (yf - y0) * ny + (zf - z0) * nz;
            const double d1 = (xf - x1) * nx + (yf - y1) * ny + (zf - z1) * nz;
            const double Xpacx = xf - nx * d0, Xpacy = yf - ny * d0, Xpacz = zf - nz * d0;
            const double Xnacx = xf - nx * d1, Xnacy = yf - ny * d1, Xnacz = zf - nz * d1;
            const double delpx = Xpacx - x0, delpy = Xpacy - y0, delpz = Xpacz - z0;
            const double delnx = Xnacx - x1, delny = Xnacy - y1, delnz = Xnacz - z1;
            const double gP0x = a.gP[0][c0], gP0y = a.gP[1][c0], gP0z = a.gP[2][c0];
            const double gP1x = a.gP[0][c1], gP1y = a.gP[1][c1], gP1z = a.gP[2][c1];
            const double cell0_P = a.P[c0] + (gP0x * delpx + gP0y * delpy + gP0z * delpz);
            const double cell1_P = a.P[c1] + (gP1x * delnx + gP1y * delny + gP1z * delnz);
            const double Xpnx = Xnacx - Xpacx, Xpny = Xnacy - Xpacy, Xpnz = Xnacz - Xpacz;
            const double X2x = x1 - x0, X2y = y1 - y0, X2z = z1 - z0;
            const double A0 = a.AU[c0], A1 = a.AU[c1];
            const double ApV0 = (A0 != 0.0) ? 1.0 / A0 : 0.0;
            const double ApV1 = (A1 != 0.0) ? 1.0 / A1 : 0.0;
            double ApV = m.rho[c0] * ApV0 * l0 + m.rho[c1] * ApV1 * l1;
            const double volume_avg = m.vol[c0] * l0 + m.vol[c1] * l1;
            ApV = ApV * m.area[face] * volume_avg / (X2x * nx + X2y * ny + X2z * nz);
            const double dpx = (gP1x * l1 + gP0x * l0) * Xpnx;
            const double dpy = (gP1y * l1 + gP0y * l0) * Xpny;
            const double dpz = (gP1z * l1 + gP0z * l0) * Xpnz;
            md -= ApV * ((cell1_P - cell0_P) - dpx - dpy - dpz);
            a.mdot[face] = md;
            a.ff0[face] = -ApV;
            a.ff1[face] = -ApV;
        } else {
            const int t = ph.btype[c1 - N];
            double md = 0.0;
            if (t == INLET) {
                md = ph.rho_in * (ph.u_in * Sx + 0.0 * Sy + 0.0 * Sz);
                part[0] += md;
            } else if (t == OUTLET) {
                if (ph.mode == 1)  // zero-gradient outlet
                    md = ph.rho_in * (a.U[c0] * Sx + a.V[c0] * Sy + a.W[c0] * Sz);
                else  // the reference's fixed outlet flux (:1969-1985)
                    md = ph.rho_in * (ph.u_in * Sx + 0.0 * Sy + 0.0 * Sz);
                if (md < 0.0) md = 1e-15;
                part[1] += md;
                part[2] += m.area[face];
            }
            a.mdot[face] = md;
        }
    }
    if (publish_partials<3>(part, a.partials, a.counter, sh)) {
        double tot[3];
        reduce_partials<3>(tot, a.partials, a.counter, sh);
        if (threadIdx.x == 0) {
            FluxBalance *bal = a.balance;
            bal->flow_in = tot[0];
            bal->flow_out = tot[1];
            bal->area_out = tot[2];
            bal->fallback = tot[1] < 0.0000000001;
            bal->rate_area = -tot[0] / tot[2];
            const double msrc = a.mass_source_dev ? *a.mass_source_dev : a.mass_source_total;
            bal->outlet_scale = (ph.mode == 1 && !bal->fallback) ? (msrc - tot[0]) / tot[1] : 1.0;
        }
    }
}

// Outlet fluxes after the balance (:2049-2079; simple mode: scale so that the
// boundary fluxes balance the particle mass source).
__global__ void k_outlet_fix(Physics ph, MeshArgs m, double *__restrict__ mdot, double *U, double *V, double *W,
                             const FluxBalance *__restrict__ bal)
{
    const int i = grid_stride_start();
    if (i >= m.n_outlet) return;
    const int face = m.outlet_faces[i];
    if (bal->fallback) {
        mdot[face] = bal->rate_area * m.area[face];
        const int slot = m.fc1[face];
        if (face == ph.last_bface[slot - ph.N]) {
            U[slot] = ph.u_in;
            V[slot] = 0.0;
            W[slot] = 0.0;
        }
    } else if (ph.mode == 1) {
        mdot[face] *= bal->outlet_scale;
    }
}

// Pressure-correction rows (the S_U accumulation of calculate_mass_flux,
// :1964 and :2101, and setup_pressure_matrix, :2139-2189).
// One cell's row; returns its diagonal.
__device__ __forceinline__ double pressure_row(const Physics &ph, const MeshArgs &m, const PressureRowArgs &a, int c)
{
    const int N = ph.N;
    const unsigned own = m.own[c];
    int faces[6], nbs[6];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        faces[k] = m.sface[(size_t)k * N + c];
        nbs[k] = m.col[(size_t)k * N + c];
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        if (nbs[k] != c) continue;
        if (ph.btype[m.fc1[faces[k]] - N] == INLET) s = s - a.mdot[faces[k]];
    }
#pragma unroll
    for (int k = 0; k < 6; k++) {
        if (nbs[k] != c) continue;
        if (ph.btype[m.fc1[faces[k]] - N] == OUTLET) s -= a.mdot[faces[k]];
    }
    if (ph.mode == 1 && a.src) s += a.src[4 * (size_t)N + c];
    double diag = 0.0;
    double offv[6];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const int face = faces[k];
        offv[k] = 0.0;
        if (nbs[k] == c) continue;
        const double md = a.mdot[face];
        if ((own >> k) & 1u) {
            s -= md;
            offv[k] = a.ff1[face];
            diag -= offv[k];
        } else {
            s += md;
            offv[k] = a.ff0[face];
            diag -= offv[k];
        }
    }
    a.b[c] = s;
    a.diag[c] = diag;
#pragma unroll
    for (int k = 0; k < 6; k++) a.off[(size_t)k * N + c] = offv[k];
    if (a.f32.d32) store_fp32_row(a.f32, N, c, diag, offv);
    if (a.dir64) store_dir_row(a.code[c], offv, a.dir64, N, c, a.dir64_sym);
    return diag;
}

// With diag_max set, also max |diag| (for the scale of the FP16 copy of the
// FP32 level 0): a warp maximum, then one atomicMax per warp on the bits of
// the non-negative value; *diag_max must be zero before the launch.
__global__ void __launch_bounds__(MCB_THREADS, 4) k_pressure_rows(Physics ph, MeshArgs m, PressureRowArgs a)
{
    const int c = grid_stride_start();
    double v = 0.0;
    if (c < ph.N) v = fabs(pressure_row(ph, m, a, c));
    if (a.diag_max) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
        if ((threadIdx.x & 31) == 0 && v > 0.0)
            atomicMax((unsigned long long *)a.diag_max, (unsigned long long)__double_as_longlong(v));
    }
}

__global__ void __launch_bounds__(MCB_THREADS) k_dir_rows64(int N, const double *__restrict__ off,
                                                           const uint32_t *__restrict__ code, double *__restrict__ out,
                                                           int sym)
{
    const int c = grid_stride_start();
    if (c >= N) return;
    double offv[6];
#pragma unroll
    for (int k = 0; k < 6; k++) offv[k] = off[(size_t)k * N + c];
    store_dir_row(code[c], offv, out, N, c, sym);
}

// ------------------------------------------------------- corrector updates
// Face part of one corrector pass of calculate_pressure: mass flux += a_f
// (PP_N - PP_P) (:2402-2412) then update_mass_flux (:1812-1878).
__global__ void __launch_bounds__(MCB_THREADS, 4) k_pp_correct_faces(Physics ph, MeshArgs m, CorrectArgs a)
{
    const int N = ph.N, F = m.F;
    for (int face = grid_stride_start(); face < F; face += gridDim.x * blockDim.x) {
        const int c0 = m.fc0[face], c1 = m.fc1[face];
        if (c1 >= N) continue;
        const double fact = a.ff0[face];
        double md = a.mdot[face];
        md += (fact * (a.PP[c1] - a.PP[c0]));
        const double Sx = m.Sx[face], Sy = m.Sy[face], Sz = m.Sz[face];
        const double smag = sqrt(Sx * Sx + Sy * Sy + Sz * Sz);
        const double nx = Sx / smag, ny = Sy / smag, nz = Sz / smag;
        const double x0 = m.xc[c0], y0 = m.yc[c0], z0 = m.zc[c0];
        const double x1 = m.xc[c1], y1 = m.yc[c1], z1 = m.zc[c1];
        const double xf = m.xf[face], yf = m.yf[face], zf = m.zf[face];
        const double d0 = (xf - x0) * nx + (yf - y0) * ny + (zf - z0) * nz;
        const double d1 = (xf - x1) * nx + (yf - y1) * ny + (zf - z1) * nz;
        double Xnx = (xf - nx * d1) - x1, Xny = (yf - ny * d1) - y1, Xnz = (zf - nz * d1) - z1;
        double Xpx = (xf - nx * d0) - x0, Xpy = (yf - ny * d0) - y0, Xpz = (zf - nz * d0) - z0;
        if (fabs(Xnx) < 0.0000000000000003) Xnx = 0.0;
        if (fabs(Xny) < 0.0000000000000003) Xny = 0.0;
        if (fabs(Xnz) < 0.0000000000000003) Xnz = 0.0;
        if (fabs(Xpx) < 0.0000000000000003) Xpx = 0.0;
        if (fabs(Xpy) < 0.0000000000000003) Xpy = 0.0;
        if (fabs(Xpz) < 0.0000000000000003) Xpz = 0.0;
        const double dpx = a.gPP[0][c1] * Xnx - a.gPP[0][c0] * Xpx;
        const double dpy = a.gPP[1][c1] * Xny - a.gPP[1][c0] * Xpy;
        const double dpz = a.gPP[2][c1] * Xnz - a.gPP[2][c0] * Xpz;
        const double fc = fact * (dpx + dpy + dpz) * ph.flux_corr;
        md += fc;
        a.mdot[face] = md;
        a.fcorr[face] = fc;
    }
}

// Cell part: P += urf_p PP and u -= V/A grad(PP) (:2416-2433; every cell in
// simple mode, only cell 0 on the first call in compat mode), the next
// corrector's right-hand side from the non-orthogonal flux corrections
// (:1875-1876, simple mode), and PP = 0 (:2447-2450).
__global__ void __launch_bounds__(MCB_THREADS, 4) k_pp_correct_cells(Physics ph, MeshArgs m, CorrectArgs a,
                                                                  int correct_all, int correct_cell0)
{
    const int N = ph.N;
    const int c = grid_stride_start();
    if (c < N) {
        if (correct_all || (correct_cell0 && c == ph.cell0)) {
            const double A = a.AU[c];
            const double Ar = (A != 0.0) ? 1.0 / A : 0.0;
            const double fact = m.vol[c] * Ar;
            a.P[c] += ph.urf_p * a.PP[c];
            a.U[c] -= a.gPP[0][c] * fact;
            a.V[c] -= a.gPP[1][c] * fact;
            a.W[c] -= a.gPP[2][c] * fact;
        }
        if (a.next_rhs) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 6; k++) {
                const int face = m.sface[(size_t)k * N + c];
                const int c0 = m.fc0[face], c1 = m.fc1[face];
                if (c1 >= N) continue;
                if (c == c0)
                    s -= a.fcorr[face];
                else
                    s += a.fcorr[face];
            }
            a.next_rhs[c] = s;
        }
        a.PP[c] = 0.0;
    } else if (c < N + 6) {
        a.PP[c] = 0.0;
    }
}

// update_P (FlowSolver.inl:2292-2315): boundary pressure from the last face
// of each side.  Only the cells of those six faces need the pressure
// gradient here (get_phi_gradient(P) before it, :2454): with `nbr` given,
// each thread first computes its cell's gradient (the same least-squares
// arithmetic as k_lsq_gradients, pressure boundary rule) into gPx/gPy/gPz.
__global__ void k_update_p_boundary(Physics ph, MeshArgs m, double *P, double *gPx, double *gPy, double *gPz,
                                    const int *nbr)
{
    const int side = threadIdx.x;
    if (side >= 6) return;
    const int face = ph.last_bface[side];
    if (face < 0) return;
    const int c0 = m.fc0[face];
    if (nbr) {
        GradArgs<1> g{};
        g.phi[0] = P;
        g.gx[0] = gPx;
        g.gy[0] = gPy;
        g.gz[0] = gPz;
        g.zero_boundary = 1u;
        lsq_cell<1>(ph.N, nbr, m.fc1, m.xc, m.yc, m.zc, m.xf, m.yf, m.zf, g, c0);
    }
    if (ph.btype[side] == OUTLET) {
        P[ph.N + side] = P[c0];
    } else {
        const double dsx = m.xf[face] - m.xc[c0], dsy = m.yf[face] - m.yc[c0], dsz = m.zf[face] - m.zc[c0];
        P[ph.N + side] = P[c0] + (gPx[c0] * dsx + gPy[c0] * dsy + gPz[c0] * dsz);
    }
}

// Largest pressure correction, as the reference computes it (:2371-2378):
// max(PP[0], max_{i >= 1} |PP[i]|), cell 0 in the reference's numbering.
__global__ void __launch_bounds__(MCB_THREADS) k_pp_max(int N, int cell0, const double *__restrict__ PP, double *partials,
                                                        unsigned int *counter, double *out)
{
    __shared__ double sh[1][MCB_THREADS];
    double v[1] = {-1.0e308};
    for (int i = grid_stride_start(); i < N; i += gridDim.x * blockDim.x) v[0] = fmax(v[0], i == cell0 ? PP[i] : fabs(PP[i]));
    if (publish_partials<1, true>(v, partials, counter, sh)) {
        double tot[1];
        reduce_partials<1, true>(tot, partials, counter, sh);
        if (threadIdx.x == 0) *out = tot[0];
    }
}

// max over cells of |net outflow - mass source| (a diagnostic of the pass).
__global__ void __launch_bounds__(MCB_THREADS) k_sum(int n, const double *__restrict__ x, double *partials,
                                                     unsigned int *counter, double *out)
{
    __shared__ double sh[1][MCB_THREADS];
    double acc[1] = {0.0};
    for (int i = grid_stride_start(); i < n; i += gridDim.x * blockDim.x) acc[0] += x[i];
    if (publish_partials<1>(acc, partials, counter, sh)) {
        double tot[1];
        reduce_partials<1>(tot, partials, counter, sh);
        if (threadIdx.x == 0) *out = tot[0];
    }
}

} // namespace mcb
