// Adjoint of the marker step with respect to the initial marker temperatures and
// the amplitudes of velocity modes, v = sum_m a_m (vx_m, vy_m).
//
// Forward model (what i2g_adjoint_forward runs): nsteps x {movemark; ronurecalc}
// with the combined velocity field, positions checkpointed (by caller index)
// every k steps.  Loss gradient dL/dtk is given at the final node temperatures
// tk = sum_i w_i T_i / sum_i w_i (markmart.c:899-906, 988-991).
//
// Reverse:
//   k_adj_avg   per marker: dL/dT_i = sum_n g_n w_in / W_n and
//               dL/dx_i = sum_n g_n (T_i - tk_n) / W_n dw_in/dx_i over its 2x2
//               nodes; temperatures the step replaced (sticky air, out of box)
//               get zero.
//   k_adj_rk4   per marker, independent of every other marker: for each
//               checkpoint segment, last first, recompute the segment's positions
//               with the forward's own arithmetic, then run the reverse of the
//               classical RK4 stage chain, using the bilinear Jacobian of the
//               velocity at every stage point and the mode velocities for
//               dL/da; per-CTA partial sums of dL/da, folded in a fixed order.
// The interpolants are piecewise bilinear; derivatives are those of the piece
// the forward used (the stencil switches at faces and midpoints have measure zero).
#pragma once

#include "i2g_kernels.cuh"

namespace i2g {

constexpr int kMaxModes = 16;
constexpr int kMaxCkptSeg = 16;  // steps per checkpoint segment held in registers

struct AdjView {
    const double *mvx, *mvy;  // [nn][nmodes] unit-amplitude mode velocities, interleaved
    int32_t nmodes;
};

// velocity at (x, y) with the forward's arithmetic, its Jacobian d(vx,vy)/d(x,y)
// and the mode velocities at the same weights
template <bool MIXED>
__device__ __forceinline__ void interp_vjac(const GridView &G, const AdjView &Md, double x, double y, double &vx,
                                            double &vy, double J[2][2], double *Vx, double *Vy)
{
    const double xc = x, yc = y;
    clampxy(G, x, y);
    const double dcx = (x == xc) ? 1.0 : 0.0, dcy = (y == yc) ? 1.0 : 0.0;  // clamped: no dependence
    const int nm = Md.nmodes;
    const int64_t ny = G.ny;
    int64_t ax, ay, bx, by;  // vx stencil (ax, ay), vy stencil (bx, by)
    double wxa0, wxa1, wya0, wya1, dxa, dya;  // vx weights and d(w1)/dx, d(w1)/dy
    double wxb0, wxb1, wyb0, wyb1, dxb, dyb;  // vy weights
    if (!MIXED) {
        const int64_t m10 = cell_search(G.gx, G.nx, G.inv_x, x), m20 = cell_search(G.gy, ny, G.inv_y, y);
        int64_t m2 = m20;
        if (y < __ldg(G.ymid + m20)) m2 -= 1;
        if (m2 < 0) m2 = 0;
        if (m2 > ny - 3) m2 = ny - 3;
        int64_t m1 = m10;
        if (x < __ldg(G.xmid + m10)) m1 -= 1;
        if (m1 < 0) m1 = 0;
        if (m1 > G.nx - 3) m1 = G.nx - 3;
        const double gx0 = __ldg(G.gx + m10), gx1 = __ldg(G.gx + m10 + 1);
        const double ym0 = __ldg(G.ymid + m2), ym1 = __ldg(G.ymid + m2 + 1);
        fdw64(gx0, gx1, x, wxa0, wxa1);
        fdw64(ym0, ym1, y, wya0, wya1);
        dxa = 1.0 / (gx1 - gx0);
        dya = 1.0 / (ym1 - ym0);
        const double xm0 = __ldg(G.xmid + m1), xm1 = __ldg(G.xmid + m1 + 1);
        const double gy0 = __ldg(G.gy + m20), gy1 = __ldg(G.gy + m20 + 1);
        fdw64(xm0, xm1, x, wxb0, wxb1);
        fdw64(gy0, gy1, y, wyb0, wyb1);
        dxb = 1.0 / (xm1 - xm0);
        dyb = 1.0 / (gy1 - gy0);
        ax = m10; ay = m2; bx = m1; by = m20;
        vx = bil64(G.vx, ny, ax, ay, wxa0, wxa1, wya0, wya1);
        vy = bil64(G.vy, ny, bx, by, wxb0, wxb1, wyb0, wyb1);
    } else {
        AxisF X, Y;
        axis_fast(G.gx, G.lx, G.nx, G.inv_x, x, -1, X);
        axis_fast(G.gy, G.ly, ny, G.inv_y, y, -1, Y);
        vx = (double)bil32i(G.vxf, (int)ny, X.b, Y.m, X.b0, X.b1, Y.m0, Y.m1);
        vy = (double)bil32i(G.vyf, (int)ny, X.m, Y.b, X.m0, X.m1, Y.b0, Y.b1);
        ax = X.b; ay = Y.m; bx = X.m; by = Y.b;
        wxa0 = X.b0; wxa1 = X.b1; wya0 = Y.m0; wya1 = Y.m1;
        wxb0 = X.m0; wxb1 = X.m1; wyb0 = Y.b0; wyb1 = Y.b1;
        dxa = __ldg(G.lx + X.b).y;
        dya = (Y.m == Y.b) ? __ldg(G.ly + Y.b).z : __ldg(G.ly + Y.m).z;
        dxb = (X.m == X.b) ? __ldg(G.lx + X.b).z : __ldg(G.lx + X.m).z;
        dyb = __ldg(G.ly + Y.b).y;
    }
    // corner values (FP64 grids for the derivatives in both forms)
    const double *pa = G.vx + ax * ny + ay, *pb = G.vy + bx * ny + by;
    const double a00 = __ldg(pa), a01 = __ldg(pa + 1), a10 = __ldg(pa + ny), a11 = __ldg(pa + ny + 1);
    const double b00 = __ldg(pb), b01 = __ldg(pb + 1), b10 = __ldg(pb + ny), b11 = __ldg(pb + ny + 1);
    J[0][0] = dcx * dxa * (wya0 * (a10 - a00) + wya1 * (a11 - a01));
    J[0][1] = dcy * dya * (wxa0 * (a01 - a00) + wxa1 * (a11 - a10));
    J[1][0] = dcx * dxb * (wyb0 * (b10 - b00) + wyb1 * (b11 - b01));
    J[1][1] = dcy * dyb * (wxb0 * (b01 - b00) + wxb1 * (b11 - b10));
    const double ca00 = wxa0 * wya0, ca01 = wxa0 * wya1, ca10 = wxa1 * wya0, ca11 = wxa1 * wya1;
    const double cb00 = wxb0 * wyb0, cb01 = wxb0 * wyb1, cb10 = wxb1 * wyb0, cb11 = wxb1 * wyb1;
    const double *ma = Md.mvx + (ax * ny + ay) * nm, *mb = Md.mvy + (bx * ny + by) * nm;
    for (int m = 0; m < nm; m++) {
        Vx[m] = ca00 * __ldg(ma + m) + ca01 * __ldg(ma + nm + m) + ca10 * __ldg(ma + ny * nm + m) +
                ca11 * __ldg(ma + (ny + 1) * nm + m);
        Vy[m] = cb00 * __ldg(mb + m) + cb01 * __ldg(mb + nm + m) + cb10 * __ldg(mb + ny * nm + m) +
                cb11 * __ldg(mb + (ny + 1) * nm + m);
    }
}

// one forward step of a marker exactly as movemark() moves it (velocity only)
template <bool MIXED>
__device__ __forceinline__ void rk4_forward(const GridView &G, const MoveArgs &A, double &x, double &y)
{
    double vx0, vy0;
    const double dt = A.timestep;
    if (MIXED) {
        int hx, hy;
        rk4_mixed(G, x, y, dt, A.markmod, vx0, vy0, nullptr, hx, hy);
    } else {
        if (A.markmod == 1) {
            interp_v<false>(G, x, y, vx0, vy0);
        } else {
            double vx1, vy1, vx2, vy2, vx3, vy3, vx4, vy4;
            interp_v<false>(G, x, y, vx1, vy1);
            interp_v<false>(G, x + vx1 * dt / 2.0, y + vy1 * dt / 2.0, vx2, vy2);
            interp_v<false>(G, x + vx2 * dt / 2.0, y + vy2 * dt / 2.0, vx3, vy3);
            interp_v<false>(G, x + vx3 * dt, y + vy3 * dt, vx4, vy4);
            vx0 = (vx1 + 2.0 * vx2 + 2.0 * vx3 + vx4) / 6.0;
            vy0 = (vy1 + 2.0 * vy2 + 2.0 * vy3 + vy4) / 6.0;
        }
    }
    if (A.outgrid == 2) {
        if (x < 0 || x > G.xsize) vy0 = 0;
        if (y < 0 || y > G.ysize) vx0 = 0;
    }
    x += dt * vx0;
    y += dt * vy0;
}

// reverse of one step: lam (dL/dx after the step) -> dL/dx before it; da += dL/da
template <bool MIXED>
__device__ __forceinline__ void rk4_reverse(const GridView &G, const AdjView &Md, const MoveArgs &A, double x,
                                            double y, double &lx, double &ly, double *da)
{
    const double dt = A.timestep;
    const int nm = Md.nmodes;
    double J[2][2], Vx[kMaxModes], Vy[kMaxModes];
    double ox = 1.0, oy = 1.0;  // orthogonal-only motion outside the box (markmart.c:100-105)
    if (A.outgrid == 2) {
        if (x < 0 || x > G.xsize) oy = 0.0;
        if (y < 0 || y > G.ysize) ox = 0.0;
    }
    // dL/d(vx0, vy0) of x' = x + dt*v0
    const double g0x = lx * dt * ox, g0y = ly * dt * oy;
    if (A.markmod == 1) {
        double vx, vy;
        interp_vjac<MIXED>(G, Md, x, y, vx, vy, J, Vx, Vy);
        for (int m = 0; m < nm; m++) da[m] += g0x * Vx[m] + g0y * Vy[m];
        lx += g0x * J[0][0] + g0y * J[1][0];
        ly += g0x * J[0][1] + g0y * J[1][1];
        return;
    }
    // stage points (recomputed with the forward's arithmetic)
    double v1x, v1y, v2x, v2y, v3x, v3y, v4x, v4y;
    const double p1x = x, p1y = y;
    interp_vjac<MIXED>(G, Md, p1x, p1y, v1x, v1y, J, Vx, Vy);
    const double p2x = x + v1x * dt / 2.0, p2y = y + v1y * dt / 2.0;
    interp_vjac<MIXED>(G, Md, p2x, p2y, v2x, v2y, J, Vx, Vy);
    const double p3x = x + v2x * dt / 2.0, p3y = y + v2y * dt / 2.0;
    interp_vjac<MIXED>(G, Md, p3x, p3y, v3x, v3y, J, Vx, Vy);
    const double p4x = x + v3x * dt, p4y = y + v3y * dt;
    // k4
    double k4x = g0x / 6.0, k4y = g0y / 6.0;
    double k3x = g0x / 3.0, k3y = g0y / 3.0;
    double k2x = g0x / 3.0, k2y = g0y / 3.0;
    double k1x = g0x / 6.0, k1y = g0y / 6.0;
    double px, py;
    interp_vjac<MIXED>(G, Md, p4x, p4y, v4x, v4y, J, Vx, Vy);
    for (int m = 0; m < nm; m++) da[m] += k4x * Vx[m] + k4y * Vy[m];
    px = k4x * J[0][0] + k4y * J[1][0];
    py = k4x * J[0][1] + k4y * J[1][1];
    lx += px;
    ly += py;
    k3x += dt * px;
    k3y += dt * py;
    // k3 at p3
    interp_vjac<MIXED>(G, Md, p3x, p3y, v3x, v3y, J, Vx, Vy);
    for (int m = 0; m < nm; m++) da[m] += k3x * Vx[m] + k3y * Vy[m];
    px = k3x * J[0][0] + k3y * J[1][0];
    py = k3x * J[0][1] + k3y * J[1][1];
    lx += px;
    ly += py;
    k2x += dt / 2.0 * px;
    k2y += dt / 2.0 * py;
    // k2 at p2
    interp_vjac<MIXED>(G, Md, p2x, p2y, v2x, v2y, J, Vx, Vy);
    for (int m = 0; m < nm; m++) da[m] += k2x * Vx[m] + k2y * Vy[m];
    px = k2x * J[0][0] + k2y * J[1][0];
    py = k2x * J[0][1] + k2y * J[1][1];
    lx += px;
    ly += py;
    k1x += dt / 2.0 * px;
    k1y += dt / 2.0 * py;
    // k1 at p1
    interp_vjac<MIXED>(G, Md, p1x, p1y, v1x, v1y, J, Vx, Vy);
    for (int m = 0; m < nm; m++) da[m] += k1x * Vx[m] + k1y * Vy[m];
    lx += k1x * J[0][0] + k1y * J[1][0];
    ly += k1x * J[0][1] + k1y * J[1][1];
}

// averaging adjoint at the final positions (device order); outputs by caller index
template <bool MIXED>
__global__ void __launch_bounds__(256) k_adj_avg(const __grid_constant__ GridView G,
                                                 const __grid_constant__ MarkerView M, const DevTypes *__restrict__ Ty,
                                                 int32_t gridmod, double tmp_ambient, const double *__restrict__ tk,
                                                 const double *__restrict__ w1, const double *__restrict__ g,
                                                 const double *__restrict__ T0, double2 *__restrict__ lam,
                                                 double *__restrict__ dT)
{
    const i2g_types &T = Ty->t;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t ny = G.ny;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < M.n; j += stride) {
        const int32_t id = M.id[j];
        const double x = M.x[j], y = M.y[j], Tm = M.T[j];
        const int mt = M.type[j];
        double gT = 0.0, gx = 0.0, gy = 0.0;
        const bool valid = x > 0 && y > 0 && x < G.xsize && y < G.ysize && Tm > 0 && mt < 50 &&
                           (gridmod <= 1 || (id % gridmod) == 0) && !T.markim[mt];
        if (valid) {
            const int64_t m10 = cell_search(G.gx, G.nx, G.inv_x, x), m20 = cell_search(G.gy, ny, G.inv_y, y);
            double wx0, wx1, wy0, wy1, ix, iy;
            if (!MIXED) {
                fdw64(__ldg(G.gx + m10), __ldg(G.gx + m10 + 1), x, wx0, wx1);
                fdw64(__ldg(G.gy + m20), __ldg(G.gy + m20 + 1), y, wy0, wy1);
                ix = 1.0 / (__ldg(G.gx + m10 + 1) - __ldg(G.gx + m10));
                iy = 1.0 / (__ldg(G.gy + m20 + 1) - __ldg(G.gy + m20));
            } else {
                float a0, a1, b0, b1;
                fdw32(__ldg(G.gx + m10), __ldg(G.ixb + m10), x, a0, a1);
                fdw32(__ldg(G.gy + m20), __ldg(G.iyb + m20), y, b0, b1);
                wx0 = a0; wx1 = a1; wy0 = b0; wy1 = b1;
                ix = __ldg(G.ixb + m10);
                iy = __ldg(G.iyb + m20);
            }
            const double wx[2] = {wx0, wx1}, wy[2] = {wy0, wy1}, dwx[2] = {-ix, ix}, dwy[2] = {-iy, iy};
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) {
                    const int64_t m3 = (m10 + a) * ny + m20 + b;
                    const double W = w1[m3];
                    if (!(W > 0)) continue;
                    const double c = g[m3] / W, r = Tm - tk[m3];
                    gT += c * wx[a] * wy[b];
                    gx += c * r * dwx[a] * wy[b];
                    gy += c * r * wx[a] * dwy[b];
                }
        }
        // temperatures replaced by the step (sticky air, out of the box) carry no gradient
        const bool replaced = mt < 2 || Tm != T0[id];
        dT[id] = replaced ? 0.0 : gT;
        lam[id] = make_double2(gx, gy);
    }
}

// reverse through all steps, one thread per marker (caller index)
template <bool MIXED>
__global__ void __launch_bounds__(128) k_adj_rk4(const __grid_constant__ GridView G, const __grid_constant__ AdjView Md,
                                                 const __grid_constant__ MoveArgs A, const DevTypes *__restrict__ Ty,
                                                 const int8_t *__restrict__ type_by_id, const double2 *__restrict__ ck,
                                                 int64_t n, int32_t nsteps, int32_t every, double2 *__restrict__ lam,
                                                 double *__restrict__ dapart)
{
    const i2g_types &T = Ty->t;
    const int nm = Md.nmodes;
    double da[kMaxModes];
    for (int m = 0; m < kMaxModes; m++) da[m] = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double2 l = lam[i];
        double lx = l.x, ly = l.y;
        const int mt = type_by_id[i];
        const int nseg = (nsteps + every - 1) / every;
        for (int sg = nseg - 1; sg >= 0; sg--) {
            const int s0 = sg * every, len = min(every, nsteps - s0);
            double xs[kMaxCkptSeg], ys[kMaxCkptSeg];
            double2 p = ck[(int64_t)sg * n + i];
            double x = p.x, y = p.y;
            for (int s = 0; s < len; s++) {
                xs[s] = x;
                ys[s] = y;
                const bool inbox = (x >= 0 && y >= 0 && x <= G.xsize && y <= G.ysize);
                if ((inbox || A.outgrid != 1) && !T.markim[mt]) rk4_forward<MIXED>(G, A, x, y);
            }
            for (int s = len - 1; s >= 0; s--) {
                const double xx = xs[s], yy = ys[s];
                const bool inbox = (xx >= 0 && yy >= 0 && xx <= G.xsize && yy <= G.ysize);
                if ((inbox || A.outgrid != 1) && !T.markim[mt]) rk4_reverse<MIXED>(G, Md, A, xx, yy, lx, ly, da);
            }
        }
        lam[i] = make_double2(lx, ly);
    }
    // per-CTA partial sums of dL/da (fixed tree order: deterministic)
    __shared__ double red[kMaxModes][128];
    for (int m = 0; m < nm; m++) red[m][threadIdx.x] = da[m];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int m = 0; m < nm; m++) red[m][threadIdx.x] += red[m][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int m = 0; m < nm; m++) dapart[(int64_t)blockIdx.x * nm + m] = red[m][0];
}

}  // namespace i2g
