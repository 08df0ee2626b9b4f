// press.cuh -- batched tridiagonal pressure solve and the streaming (elementwise)
// kernels of the hot path.
#pragma once
#include "fft.cuh"

namespace obl {

template <typename T> struct TdmaArgs {
    const C2<T> *Hx, *Hy, *Hz;  // spectral planes (lhx, nyt) of levels 0..nz (Hx,Hy use 1..L)
    C2<T> *phat;                // out: levels 0..L
    C2<T> *dph;                 // optional out: (p_hat(z) - p_hat(z-1))/dz at levels 1..L,
                                // formed in the solve's precision (the spectrum of dpdz)
    T *cscr;                    // bulk scratch: modified upper band c'(1..L), (S, L)
    const double *kx;           // kx(lhx), Nyquist entry 0       (002_fft.f90:131-137)
    const double *ky;           // ky_2d row (nyt), Nyquist row 0 (002_fft.f90:147,161-165)
    const unsigned char *skip;  // optional: 1 = column solved by the FP64 island kernel
    long long S;                // lhx * nyt
    int lhx, nyt, L;
    double dz;
    int neumann_top;            // OBL_TOP_NEUMANN
    // G form (gform = 1): Hx holds the y-transform of G = i*kx*H_x + (H_z(z+1) - H_z(z)
    // [+ H_z(0) at z = 1])/dz, formed before the transform (kx and the z-difference are
    // constant along y); H_z is transformed at level 0 and, at levels 1..L, only in the
    // line group of kx = 0 (the (0,0) mode's RHS).  The RHS is then G + i*ky*H_y.
    int gform;
};

// FP64 island work list
struct IslandArgs {
    const int *cols;   // column indices q = kx + lhx*ky
    int n;
    double *cscr;      // (n, L)
    double2 *dscr;     // (n, L+1)
};

// levels the solve's loads run ahead of its recurrence
#ifndef OBL_TDMA_AHEAD
#define OBL_TDMA_AHEAD 4
#endif
constexpr int kTdmaAhead = OBL_TDMA_AHEAD;

// One column's solve; t = the thread's index among the bulk columns or in the island list.
template <typename TS, typename TC, bool ISLAND, bool G = false>
__device__ __forceinline__ void tdma_column(const TdmaArgs<TS> &a, const IslandArgs &isl, long long t)
{
    using CS = C2<TS>;
    using CC = C2<TC>;
    long long q;
    if constexpr (ISLAND) {
        if (t >= isl.n) return;
        q = isl.cols[t];
    } else {
        if (t >= a.S) return;
        q = t;
        if (a.skip && a.skip[q]) return;
    }
    const long long S = a.S;
    const int L = a.L;
    const int ix = (int)(q % a.lhx), iy = (int)(q / a.lhx);
    CS *ph = a.phat + q;

    // Nyquist columns: p_hat = 0 at every level (:303-305, and the caller's zero fill)
    if (ix == a.lhx - 1 || iy == a.nyt / 2) {
        for (int z = 0; z <= L; ++z) ph[S * z] = mk<TS>(0, 0);
        if (a.dph)
            for (int z = 1; z <= L; ++z) a.dph[q + S * z] = mk<TS>(0, 0);
        return;
    }
    const double kxd = a.kx[ix], kyd = a.ky[iy];
    const double k2d = kxd * kxd + kyd * kyd;   // 002_fft.f90:167
    const bool m00 = (k2d == 0.0);              // the (0,0) mean mode
    const TC kx = (TC)kxd, ky = (TC)kyd, k2 = (TC)k2d;
    const TC dz = (TC)a.dz, idz = (TC)(1.0 / a.dz), idz2 = (TC)(1.0 / (a.dz * a.dz));

    auto ld = [&](const CS *p, int z) -> CC {
        const CS v = p[q + S * z];
        return mk<TC>((TC)v.x, (TC)v.y);
    };
    auto st_d = [&](int z, CC v) {
        if constexpr (ISLAND) isl.dscr[t + (long long)isl.n * z] = make_double2(v.x, v.y);
        else ph[S * z] = v;
    };
    auto ld_d = [&](int z) -> CC {
        if constexpr (ISLAND) { const double2 v = isl.dscr[t + (long long)isl.n * z]; return mk<TC>(v.x, v.y); }
        else return ph[S * z];
    };
    auto st_c = [&](int z, TC v) {
        if constexpr (ISLAND) isl.cscr[t + (long long)isl.n * (z - 1)] = v;
        else a.cscr[q + S * (z - 1)] = v;
    };
    auto ld_c = [&](int z) -> TC {
        if constexpr (ISLAND) return isl.cscr[t + (long long)isl.n * (z - 1)];
        else return a.cscr[q + S * (z - 1)];
    };

    // ---- forward elimination ----
    // The sweep is latency-bound: every column of the problem is in flight at once, so the
    // time per level is the load latency divided by how far ahead the loads run.  The RHS
    // inputs of the next kTdmaAhead levels are kept in a ring of registers (storage type):
    // slot s holds level base+s, refilled with level base+s+kTdmaAhead as soon as it is used.
    constexpr int PF = kTdmaAhead;
    using CS2 = C2<TS>;
    auto raw = [&](const CS *p, int z) -> CS2 { return p[q + S * z]; };
    auto cv = [&](CS2 v) -> CC { return mk<TC>((TC)v.x, (TC)v.y); };
    const CC hz0 = ld(a.Hz, 0);     // RHS_col(0) = H_z(0) (:209)
    CS2 rx[PF], ry[PF], rz[PF];
#pragma unroll
    for (int s = 0; s < PF; ++s) {
        const int z = 1 + s;
        rx[s] = raw(a.Hx, z <= L ? z : L);
        ry[s] = raw(a.Hy, z <= L ? z : L);
        if constexpr (!G) rz[s] = raw(a.Hz, z <= L + 1 ? z : L + 1);
    }
    CC dprev = hz0;
    TC cprev = 0;                   // coef_cp(0) = 0 on the bottom rank
    for (int base = 1; base <= L; base += PF) {
#pragma unroll
        for (int s = 0; s < PF; ++s) {
            const int iz = base + s;
            if (iz > L) break;
            const CC hx = cv(rx[s]), hy = cv(ry[s]);
            CC hzc = mk<TC>(0, 0), hzn = mk<TC>(0, 0);
            if constexpr (!G) {
                hzc = cv(rz[s]);
                hzn = cv(rz[(s + 1) % PF]);   // level iz+1 (slot 0 was refilled at s = 0)
            }
            {
                const int zn = iz + PF;
                rx[s] = raw(a.Hx, zn <= L ? zn : L);
                ry[s] = raw(a.Hy, zn <= L ? zn : L);
                if constexpr (!G) rz[s] = raw(a.Hz, zn <= L + 1 ? zn : L + 1);
            }
            TC am, bm, cm;
            CC r;
            if (!m00) {
                const bool top = a.neumann_top && iz == L;
                am = (iz == 1) ? (TC)0 : idz2;
                bm = (iz == 1 || top) ? -(k2 + idz2) : -(k2 + (TC)2 * idz2);
                cm = top ? (TC)0 : idz2;
                if constexpr (G) {
                    r = mk<TC>(hx.x - ky * hy.y, hx.y + ky * hy.x);   // G + i*ky*H_y
                } else {
                    const CC sxy = mk<TC>(kx * hx.x + ky * hy.x, kx * hx.y + ky * hy.y);
                    CC dh = csub(hzn, hzc);
                    if (iz == 1) dh = cadd(dh, hz0);
                    r = mk<TC>(-sxy.y + dh.x / dz, sxy.x + dh.y / dz);
                }
            } else {
                am = (iz == 1) ? (TC)0 : -idz;
                bm = idz;
                cm = 0;
                if constexpr (G) {
                    r = (iz == 1) ? mk<TC>(0, 0) : cv(raw(a.Hz, iz));   // q = 0: the (0,0) mode
                } else {
                    r = (iz == 1) ? mk<TC>(0, 0) : hzc;
                }
            }
            const TC bp = bm - am * cprev;
            const TC ibp = (TC)1 / bp;
            const TC cp = cm * ibp;
            const CC d = mk<TC>((r.x - am * dprev.x) * ibp, (r.y - am * dprev.y) * ibp);
            st_c(iz, cp);
            st_d(iz, d);
            cprev = cp;
            dprev = d;
        }
    }
    // ---- back substitution ----
    // the same ring for d(iz), c'(iz), iz = L-1 down to 1; the rows read ahead are below
    // the ones already overwritten with p_hat, so the read-ahead never sees a p value
    CC pn = a.neumann_top ? dprev : mk<TC>(0, 0);   // p_hat(nz-1): solved row / forced 0
    ph[S * L] = mk<TS>((TS)pn.x, (TS)pn.y);
    C2<TS> *dph = a.dph ? a.dph + q : nullptr;
    const TC rdz = (TC)(1.0 / a.dz);
    CC rd[PF];
    TC rc[PF];
#pragma unroll
    for (int s = 0; s < PF; ++s) {
        const int z = L - 1 - s;
        rd[s] = z >= 1 ? ld_d(z) : mk<TC>(0, 0);
        rc[s] = z >= 1 ? ld_c(z) : (TC)0;
    }
    for (int base = L - 1; base >= 1; base -= PF) {
#pragma unroll
        for (int s = 0; s < PF; ++s) {
            const int iz = base - s;
            if (iz < 1) break;
            const CC d = rd[s];
            const TC cp = rc[s];
            const int zn = iz - PF;
            if (zn >= 1) {
                rd[s] = ld_d(zn);
                rc[s] = ld_c(zn);
            }
            const CC p = mk<TC>(d.x - cp * pn.x, d.y - cp * pn.y);
            if (dph) dph[S * (iz + 1)] = mk<TS>((TS)((pn.x - p.x) * rdz), (TS)((pn.y - p.y) * rdz));
            ph[S * iz] = mk<TS>((TS)p.x, (TS)p.y);
            pn = p;
        }
    }
    // Neumann ghost level below the wall (:313-315)
    const CC p0 = mk<TC>(pn.x - dz * hz0.x, pn.y - dz * hz0.y);
    ph[0] = mk<TS>((TS)p0.x, (TS)p0.y);
    if (dph) dph[S] = mk<TS>((TS)((pn.x - p0.x) / dz), (TS)((pn.y - p0.y) / dz));
}

// (a.gform selects the G-form instantiations of the solves)
template <typename T> void launch_tdma(const TdmaArgs<T> &a, cudaStream_t s, cudaError_t &e);
// the G form's y-transform of G into Hx (levels 1..L, in place)
template <typename T>
cudaError_t launch_gform_cols(int ny, C2<T> *Hx, const C2<T> *Hz, const double *kx, long long S, int lhx, int L,
                              double dz, const C2<T> *twF, cudaStream_t s);
// FP32 bulk columns by the register-segmented partitioned solve (no scratch traffic),
// FP64 island columns (isl.n may be 0) by the sequential FP64 sweep in the same launch;
// levels L <= 256
bool tdma_reg_supported(int L);
// the same solve as a persistent kernel fed by bulk asynchronous copies (FP32 storage, the
// three-spectra RHS); ctl: device ints {work counter, error flag}, the flag set to 1 when a
// bounded wait gave up; extra_tx: 0 (a test sets bytes that never arrive)
bool tdma_staged_supported(const TdmaArgs<float> &a);
void launch_tdma_staged(const TdmaArgs<float> &a, const IslandArgs &isl, int *ctl, unsigned extra_tx, cudaStream_t s,
                        cudaError_t &e);
template <typename T> void launch_tdma_reg(const TdmaArgs<T> &a, const IslandArgs &isl, cudaStream_t s,
                                           cudaError_t &e);
template <typename T> void launch_tdma_island(const TdmaArgs<T> &a, const IslandArgs &isl,
                                              cudaStream_t s, cudaError_t &e);

// streaming kernels on (ldx, nyt, levels) fields
template <typename T> void launch_ddz_uv(T *dfdz, const T *fun, int nxt, int ldx, int nyt, int nz,
                                         double dz, cudaStream_t s, cudaError_t &e);
template <typename T> void launch_ddz_w(T *dfdz, const T *fun, int nxt, int ldx, int nyt, int nz,
                                        double dz, cudaStream_t s, cudaError_t &e);
template <typename T> void launch_dpdz(T *dpdz, const T *p, int nxt, int ldx, int nyt, int nz,
                                       double dz, cudaStream_t s, cudaError_t &e);
// only the boundary part of project (110_project.f90:50-60), after an interior update
template <typename T> void launch_project_bc(T *u, T *v, T *w, int ldx, int nyt, int nz, int stress_free,
                                             cudaStream_t s, cudaError_t &e);
template <typename T> void launch_project(T *u, T *v, T *w, const T *dpdx, const T *dpdy,
                                          const T *dpdz, int nxt, int ldx, int nyt, int nz,
                                          double dt, int stress_free, cudaStream_t s,
                                          cudaError_t &e);
void launch_convert_d2f(float *dst, const double *src, long long n, cudaStream_t s, cudaError_t &e);
void launch_convert_f2d(double *dst, const float *src, long long n, cudaStream_t s, cudaError_t &e);

} // namespace obl
