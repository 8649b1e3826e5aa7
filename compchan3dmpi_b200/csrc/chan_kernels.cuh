// chan_kernels.cuh -- sm_100a kernels of the compressible-channel time step.
//
// Device layout (all FP64):
//   Q  [5][nP3+2][nP2+2][px]   conservative state rho,rho*u,rho*v,rho*w,rho*E.
//                              Indices equal the reference's solV(0:nP1+1,
//                              0:nP2+1,0:nP3+1,1:5) (v1.10/codes/main_v1.9.f90:43).
//                              The 2-deep periodic ghosts are written by the
//                              stage kernel itself, so every read is plain.
//   WP [2][8][nP2+2][px]       primitive state of the two wall planes k=1, k=nP3:
//                              rho,u,v,w,E,T,p,mu.  The wall pressure is a
//                              state variable of its own (pressure BC).
//   CS [nP3+2][4][7]           var at the four periodic corner columns.  The
//                              reference never refreshes these (its halo
//                              datatypes skip corners), yet its plane
//                              statistics sum them; kept only for that.
//
// One RK stage = k_stage (fluxes + update, fused) + k_wall (wall BC +
// pressure BC).  k_stats_part + k_stats_fin run every istat steps.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace chan {

// Step counter and time of the step being computed, kept on the device for
// launches replayed from a CUDA graph (whose kernel arguments are fixed at
// capture); k_clock_advance moves it at the start of every step.
struct DevClock {
    long long step;
    double time;
};

struct DevStatus {
    int blown;             // rho<0 or T<0 seen (reference blow-up test)
    int ijk[3];            // one offending point, 1-based reference indices
    int nonfinite;         // NaN/Inf seen
    int nf_ijk[3];
    long long blown_step;  // step in which the blow-up happened
    int stall;             // 1: a stage kernel's bulk copy did not complete in time; 2: misaligned staging area
    int pad;
};

// Boundary condition of one wall plane (plug-in of the reference's wall-BC
// variants in v1.9_strat, v1.9_groov, v1.9_groov_strat, v1.9_STWNV and v1.9_RD, lines ~605-640).
struct WallBC {
    int vel;              // 0 no-slip; 1 slip mask: c0*u1+c1*u2+c2*u3 = g where mask, else no-slip;
                          // 2 prescribed (u_w, v_w) field; 3 wave v_w = A sin(k x1 + om t + ph*(j odd))
    int therm;            // 0 isothermal Tw; 1 fixed one-sided gradient c0*T1+c1*T2+c2*T3 = dTdz
    double Tw, dTdz, g;
    double A, kx, om, ph;
    const unsigned char *mask;  // [nP2][nP1], 1-based (i,j) at (j-1)*nP1 + i-1
    const double *uv;           // [2][nP2][nP1]
    const double *x1;           // [nP1] x coordinates for the wave
};

// Flux arithmetic is templated on its real type R: double for the plain FP64
// path, float for the mixed-precision path (FP32 fluxes and stage storage,
// FP64 primitive recovery, RK accumulation and reductions).  FluxC holds the
// constants the flux formulas use, in R.
template <typename R>
struct FluxC {
    R invRe, ggM, two3rd, kq, inv_gM2;
    R hdx, hdy, sx8, sx12, sy8, sy12;
    R pex, pey, PexVal, PeyVal, pez_val;
};

struct KParams {
    // geometry
    int n1, n2, n3, px, NJ, kchunk;
    long long plane, vol;
    // state: stage input and output in the stage's storage type (double, or
    // float for the intermediate stages of the mixed-precision path); the RK
    // base state is always double
    const void *qin;
    const double *qbase;
    void *qout;
    double *wp;
    const double *cs;
    // per-k tables [nP3+2]
    const double *czh;    // 0.5*invdXi*invJac(k)
    const double *cz8;    // invdXi*invJac(k)/8
    const double *cz12;   // invdXi*invJac(k)/12
    const double *pez;    // Re*dXi*jac(k)
    const float *tabf;    // the same four tables in float, [4][nP3+2] (mixed precision)
    // forcing / stats
    double *stat;         // stat1[7*n3] | stat2[7*n3] | corr[9*n3] | tau[2]
    double *tacc;         // running sums of the same 23*n3+2 numbers over statistics steps
    double *hwt;          // [4][nP2+2][px] hD on the top wall plane, staged by the last k-chunk
    DevStatus *status;
    // physics
    double invRe, ggM, ggMh, gM2, inv_gM2, kq, two3rd;
    double hdx, hdy, sx8, sx12, sy8, sy12, invdx, invdy;
    double pex, pey, pez_val;   // Re*dx, Re*dy (x,y Peclet prefactors); PezVal
    double PexVal, PeyVal;
    double inv_dz1, inv_dzN;
    double Twb, Twt, muwb, muwt;
    FluxC<double> cd;     // flux constants in double (plain FP64 path)
    FluxC<float> cf;      // and in float (mixed-precision path)
    double f1[3], f2[3], b1[3], b2[3];  // wall one-sided coefficients
    // RK stage
    double rk_a, rk_b, rk_cdt;
    int rk_mode;          // 0: in + cdt*R ; 1: base + cdt*R ; 2: a*base + b*in + cdt*R
    int check;            // last stage of a step: run the blow-up test
    int force_on;
    int acc_on;           // statistics steps also add into tacc (time averaging)
    int wall_custom;      // any wall uses a non-default WallBC
    WallBC wbc[2];
    // buoyancy body force ri*rho*(T - tref) on the wall-normal momentum and its
    // work ggM*w*(that) on the energy (a Boussinesq-style term for stratified
    // sweeps; the reference has none).  buoy_on = 0 leaves the RHS unchanged.
    double ri, tref;
    int buoy_on;
    double time;          // time of the step being computed (the reference's `time`)
    long long step;       // step number being computed
    const DevClock *clk;  // non-null in graph replays: step and time come from here
};

// step / time of the step being computed (kernel argument, or the device clock)
__device__ __forceinline__ long long kstep(const KParams &P) { return P.clk ? P.clk->step : P.step; }
__device__ __forceinline__ double ktime(const KParams &P) { return P.clk ? P.clk->time : P.time; }

__device__ __forceinline__ bool frozen(const DevStatus *st, long long step)
{
    // after a blow-up the reference stops; later steps do nothing here
    volatile const DevStatus *v = st;
    return v->blown && v->blown_step < step;
}

__device__ __forceinline__ void flag_blown(DevStatus *st, int i, int j, int k, long long step)
{
    if (atomicCAS(&st->blown, 0, 1) == 0) {
        st->ijk[0] = i; st->ijk[1] = j; st->ijk[2] = k;
        st->blown_step = step;
    }
}

__device__ __forceinline__ void flag_nonfinite(DevStatus *st, int i, int j, int k)
{
    if (atomicCAS(&st->nonfinite, 0, 1) == 0) {
        st->nf_ijk[0] = i; st->nf_ijk[1] = j; st->nf_ijk[2] = k;
    }
}

// ---------------------------------------------------------------------------
// Inviscid stencil weights.  Both branches of the reference's hybrid scheme are
// linear in the conservative variable once the velocities are fixed, so a
// point's flux derivative along one axis is sum_m w[m]*Q(offset m-2) with
// weights shared by all five variables.
//  central : (-u2 Q2 + 8 u1 Q1 - 8 u-1 Q-1 + u-2 Q-2) /(12 d)   main_v1.9.f90:364-368
//  QUICK   : ue*Qe - uw*Qw, face values upwinded on the face velocity sign,
//            the four sign branches of main_v1.9.f90:335-361
template <typename R>
__device__ __forceinline__ void quick_weights(R um1, R u0, R up1, R s8, R w[5])
{
    const R r1 = (u0 + up1) * R(0.5);  // tmpR1, east face
    const R r2 = (u0 + um1) * R(0.5);  // tmpR2, west face
    const bool e = r1 >= R(0), f = r2 >= R(0);
    const R R1 = r1 * s8, R2 = r2 * s8;
    // east face value at offsets -1,0,+1,+2 ; west face at -2,-1,0,+1
    const R ae_m1 = e ? R(-1) : R(0), ae_0 = e ? R(6) : R(3), ae_1 = e ? R(3) : R(6), ae_2 = e ? R(0) : R(-1);
    const R bw_m2 = f ? R(-1) : R(0), bw_m1 = f ? R(6) : R(3), bw_0 = f ? R(3) : R(6), bw_1 = f ? R(0) : R(-1);
    w[0] = -R2 * bw_m2;
    w[1] = R1 * ae_m1 - R2 * bw_m1;
    w[2] = R1 * ae_0 - R2 * bw_0;
    w[3] = R1 * ae_1 - R2 * bw_1;
    w[4] = R1 * ae_2;
}

template <typename R>
__device__ __forceinline__ void central_weights(R um2, R um1, R up1, R up2, R s12, R w[5])
{
    w[0] = um2 * s12;
    w[1] = R(-8) * um1 * s12;
    w[2] = R(0);
    w[3] = R(8) * up1 * s12;
    w[4] = -(up2 * s12);
}

template <typename R>
__device__ __forceinline__ void inv_weights(R um2, R um1, R u0, R up1, R up2, bool quick, R s8, R s12, R w[5])
{
    // Both weight sets, then a select per weight.  The switch differs from lane
    // to lane where the cell Peclet number crosses its limit, and a branch there
    // runs both paths one after the other (2.6% of the FP64 stage time, 1% of the
    // float one together with the top-plane hoist below).
#ifndef CHAN_INV_BRANCH
    constexpr bool sel = true;
#else
    constexpr bool sel = false;
#endif
    if (sel) {
        R a[5], b[5];
        quick_weights(um1, u0, up1, s8, a);
        central_weights(um2, um1, up1, up2, s12, b);
#pragma unroll
        for (int m = 0; m < 5; m++) w[m] = quick ? a[m] : b[m];
    } else if (quick) {
        quick_weights(um1, u0, up1, s8, w);
    } else {
        central_weights(um2, um1, up1, up2, s12, w);
    }
}

template <typename R>
__device__ __forceinline__ R wsum(const R w[5], R q0, R q1, R q2, R q3, R q4)
{
    return (((w[0] * q0 + w[1] * q1) + w[2] * q2) + w[3] * q3) + w[4] * q4;
}

// ---------------------------------------------------------------------------
// Viscous / pressure flux vectors of main_v1.9.f90:457-538 in stress form.
// fD2..fD5 (fD1 = 0).  The energy component uses the identity
//   ggM*u*p + dissF = ggM*(u*fD2 + v*fD3 + w*fD4),
// which is the reference's dissF regrouped (same terms, different rounding).
template <typename R>
struct SlotT {
    const R *U, *V, *W, *T;
};

// pressure at box point b.  With a pressure ring (PRING) PR is the ring's
// pressure slot; without one PR is the density slot and p is rho*T/(gama*Ma^2)
// formed on the spot (one multiply against two shared loads).  On interior
// planes both give the same bits in FP64: the ring's p is formed by the same
// two products of the same values.
template <typename R, bool PRING = (sizeof(R) == 8)>
__device__ __forceinline__ R pres_at(const FluxC<R> &C, const SlotT<R> &s, const R *PR, int b)
{
    if constexpr (!PRING) return (PR[b] * s.T[b]) * C.inv_gM2;
    else return PR[b];
}

// Single-rounding multiply-add in the ring type.  The viscous fluxes are
// written with explicit FMAs so that every place that evaluates one (own
// columns, halo lanes, the k-march prologue) rounds it the same way, and a
// point's result does not depend on the launch shape that computed it.
template <typename R>
__device__ __forceinline__ R fmaR(R a, R b, R c);
template <>
__device__ __forceinline__ double fmaR<double>(double a, double b, double c) { return __fma_rn(a, b, c); }
template <>
__device__ __forceinline__ float fmaR<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
// an add the compiler may not fuse with a product feeding it
template <typename R>
__device__ __forceinline__ R addR(R a, R b);
template <>
__device__ __forceinline__ double addR<double>(double a, double b) { return __dadd_rn(a, b); }
template <>
__device__ __forceinline__ float addR<float>(float a, float b) { return __fadd_rn(a, b); }

// fD from the gradients at one point: [p + 2/3 mu/Re div - 2 mu/Re u_x,
// -mu/Re (v_x+u_y), -mu/Re (w_x+u_z), -kq mu T_x + ggM (u fD2 + v fD3 + w fD4)]
template <typename R>
__device__ __forceinline__ void fd_point(const FluxC<R> &C, R mu, R pr, R u0, R v0, R w0, R ux, R vy, R wz, R vx,
                                         R uy, R wx, R uz, R Tx, R f[4])
{
    const R mr = mu * C.invRe, kqm = C.kq * mu;
    const R div = addR(addR(ux, vy), wz);
    const R pd = fmaR(C.two3rd * mr, div, pr);
    const R t12 = mr * addR(vx, uy);
    const R f2 = fmaR(-(R(2) * mr), ux, pd);
    const R f4 = -(mr * addR(wx, uz));
    f[0] = f2;
    f[1] = -t12;
    f[2] = f4;
    f[3] = fmaR(C.ggM, fmaR(w0, f4, fmaR(u0, f2, -(v0 * t12))), -(kqm * Tx));
}

// gD from the gradients at one point (gD2 = fD3, the shared shear stress)
template <typename R>
__device__ __forceinline__ void gd_point(const FluxC<R> &C, R mu, R pr, R u0, R v0, R w0, R ux, R vy, R wz, R vx,
                                         R uy, R wy, R vz, R Ty, R g[4])
{
    const R mr = mu * C.invRe, kqm = C.kq * mu;
    const R div = addR(addR(ux, vy), wz);
    const R pd = fmaR(C.two3rd * mr, div, pr);
    const R t12 = mr * addR(vx, uy);
    const R g3 = fmaR(-(R(2) * mr), vy, pd);
    const R g4 = -(mr * addR(wy, vz));
    g[0] = -t12;
    g[1] = g3;
    g[2] = g4;
    g[3] = fmaR(C.ggM, fmaR(w0, g4, fmaR(v0, g3, -(u0 * t12))), -(kqm * Ty));
}

// The flux helpers below take plane t's primitives from the ring slot s, plane
// t+1's from sp, and plane t-1's values at point b as scalars (um, vm, wm),
// which the caller keeps outside the ring.
template <int BX, typename R, bool PRING = (sizeof(R) == 8)>
__device__ __forceinline__ void visc_fx(const FluxC<R> &C, const SlotT<R> &s, R um, R wm, const SlotT<R> &sp,
                                        const R *MU, const R *PR, int b, R czt, R f[4])
{
    const R ux = (s.U[b + 1] - s.U[b - 1]) * C.hdx;
    const R uy = (s.U[b + BX] - s.U[b - BX]) * C.hdy;
    const R vx = (s.V[b + 1] - s.V[b - 1]) * C.hdx;
    const R vy = (s.V[b + BX] - s.V[b - BX]) * C.hdy;
    const R wx = (s.W[b + 1] - s.W[b - 1]) * C.hdx;
    const R Tx = (s.T[b + 1] - s.T[b - 1]) * C.hdx;
    const R uz = (sp.U[b] - um) * czt;
    const R wz = (sp.W[b] - wm) * czt;
    fd_point(C, MU[b], pres_at<R, PRING>(C, s, PR, b), s.U[b], s.V[b], s.W[b], ux, vy, wz, vx, uy, wx, uz, Tx, f);
}

template <int BX, typename R, bool PRING = (sizeof(R) == 8)>
__device__ __forceinline__ void visc_fy(const FluxC<R> &C, const SlotT<R> &s, R vm, R wm, const SlotT<R> &sp,
                                        const R *MU, const R *PR, int b, R czt, R g[4])
{
    const R ux = (s.U[b + 1] - s.U[b - 1]) * C.hdx;
    const R uy = (s.U[b + BX] - s.U[b - BX]) * C.hdy;
    const R vx = (s.V[b + 1] - s.V[b - 1]) * C.hdx;
    const R vy = (s.V[b + BX] - s.V[b - BX]) * C.hdy;
    const R wy = (s.W[b + BX] - s.W[b - BX]) * C.hdy;
    const R Ty = (s.T[b + BX] - s.T[b - BX]) * C.hdy;
    const R vz = (sp.V[b] - vm) * czt;
    const R wz = (sp.W[b] - wm) * czt;
    gd_point(C, MU[b], pres_at<R, PRING>(C, s, PR, b), s.U[b], s.V[b], s.W[b], ux, vy, wz, vx, uy, wy, vz, Ty, g);
}

// fD and gD together at one point: they share eight gradients, the shear
// stress mu*(dv/dx+du/dy) (fD3 = gD2) and p + 2/3*mu*div.
template <int BX, typename R, bool PRING = (sizeof(R) == 8)>
__device__ __forceinline__ void visc_fxy(const FluxC<R> &C, const SlotT<R> &s, R um, R vm, R wm, const SlotT<R> &sp,
                                         const R *MU, const R *PR, int b, R czt, R f[4], R g[4])
{
    const R ux = (s.U[b + 1] - s.U[b - 1]) * C.hdx;
    const R uy = (s.U[b + BX] - s.U[b - BX]) * C.hdy;
    const R vx = (s.V[b + 1] - s.V[b - 1]) * C.hdx;
    const R vy = (s.V[b + BX] - s.V[b - BX]) * C.hdy;
    const R wx = (s.W[b + 1] - s.W[b - 1]) * C.hdx;
    const R wy = (s.W[b + BX] - s.W[b - BX]) * C.hdy;
    const R Tx = (s.T[b + 1] - s.T[b - 1]) * C.hdx;
    const R Ty = (s.T[b + BX] - s.T[b - BX]) * C.hdy;
    const R uz = (sp.U[b] - um) * czt;
    const R vz = (sp.V[b] - vm) * czt;
    const R wz = (sp.W[b] - wm) * czt;
    const R mu = MU[b], pr = pres_at<R, PRING>(C, s, PR, b);
    const R u0 = s.U[b], v0 = s.V[b], w0 = s.W[b];
    fd_point(C, mu, pr, u0, v0, w0, ux, vy, wz, vx, uy, wx, uz, Tx, f);
    gd_point(C, mu, pr, u0, v0, w0, ux, vy, wz, vx, uy, wy, vz, Ty, g);
}

template <typename R>
__device__ __forceinline__ void visc_fz_vals(const FluxC<R> &C, R ux, R vy, R wx, R wy, R u, R v, R w, R mu, R pr,
                                             R uz, R vz, R wz, R Tz, R h[4])
{
    const R mr = mu * C.invRe, kqm = C.kq * mu;
    const R div = addR(addR(ux, vy), wz);
    const R h2 = -(mr * addR(wx, uz));
    const R h3 = -(mr * addR(wy, vz));
    const R h4 = fmaR(-(R(2) * mr), wz, fmaR(C.two3rd * mr, div, pr));
    h[0] = h2;
    h[1] = h3;
    h[2] = h4;
    h[3] = fmaR(C.ggM, fmaR(w, h4, fmaR(v, h3, u * h2)), -(kqm * Tz));
}

// hD at the thread's own column; z-derivatives supplied by the caller
template <int BX, typename R>
__device__ __forceinline__ void visc_fz(const FluxC<R> &C, const SlotT<R> &s, R mu, R pr, int b, R uz, R vz, R wz,
                                        R Tz, R h[4])
{
    visc_fz_vals(C, (s.U[b + 1] - s.U[b - 1]) * C.hdx, (s.V[b + BX] - s.V[b - BX]) * C.hdy,
                 (s.W[b + 1] - s.W[b - 1]) * C.hdx, (s.W[b + BX] - s.W[b - BX]) * C.hdy, s.U[b], s.V[b], s.W[b],
                 mu, pr, uz, vz, wz, Tz, h);
}

// periodic image of index i in 0..n+1 (duplicate-point period n-2):
// q(0)=q(n-2), q(1)=q(n-1), q(n)=q(2), q(n+1)=q(3)
__device__ __forceinline__ int wrap_idx(int i, int n)
{
    if (i == 0) return n - 2;
    if (i == 1) return n - 1;
    if (i == n) return 2;
    if (i == n + 1) return 3;
    return i;
}

// ---------------------------------------------------------------------------
// Short math for the transport law mu = k = T^0.7 (main_v1.9.f90:643, 720) and
// for 1/rho.  Both start from hardware approximations and refine in FP64.
//
// The seeds are the approximations themselves: rcp.approx.ftz.f64 for the
// reciprocal, ex2.approx.ftz.f32 after lg2.approx.ftz.f32 for the power.  The FP64
// refinement squares (Newton) or cubes (Halley) the seed's relative error at
// each step, so it reaches the same accuracy from them as from exact float
// values.  Measured against the alternatives on the FP64 stage kernel: the
// correctly rounded float reciprocal __frcp_rn and the library exp2f
// (CHAN_EXACT_SEEDS) 7.5% slower; the float reciprocal approximation with its
// two conversions (CHAN_F32_RCP_SEED) 1.2% slower.
__device__ __forceinline__ float seed_rcp(float x)
{
#ifndef CHAN_EXACT_SEEDS
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return __frcp_rn(x);
#endif
}
__device__ __forceinline__ float seed_log2(float x)
{
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float seed_exp2(float x)
{
#ifndef CHAN_EXACT_SEEDS
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return exp2f(x);
#endif
}

// rcp_fast: 1/x from the seed r by one third-order step, r (1 + e + e^2) with
// e = 1 - x r (the seed's error cubed: to about 1 ulp), one dependent FMA fewer
// than two Newton steps (CHAN_RCP_NEWTON2; 0.5% of the FP64 stage time).  Valid
// for |x| in the normal range, which covers rho and mu of any physical state.
__device__ __forceinline__ double rcp_fast(double x)
{
#if !defined(CHAN_F32_RCP_SEED) && !defined(CHAN_EXACT_SEEDS)
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
#else
    double r = (double)seed_rcp((float)x);
#endif
#ifndef CHAN_RCP_NEWTON2
    // one step of third order: 1/x = r / (1 - e) = r (1 + e + e^2 + ...), e = 1 - x r
    const double e = fma(-x, r, 1.0);
    return fma(r, fma(e, e, e), r);
#else
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
#endif
}

// pow07: y = T^0.7 = T x with x = T^-0.3, the positive root of x^10 T^3 = 1.
// From the float seed x0 = exp2(-0.3 log2 T) (relative error ~3e-7),
// e = 1 - x0^10 T^3 (~3e-6) and x = x0 (1 - e)^(-1/10), whose binomial series
// 1 + e/10 + 0.055 e^2 + ... is cut after e^2 (the rest ~1e-18): twelve FP64
// operations and no division, so the result is limited by FP64 rounding
// (~2 ulp).  The earlier form, one Halley step on y^10 = T^7 with a reciprocal
// (CHAN_POW_HALLEY), takes 0.4% more of the FP64 stage time.  T <= 0 gives NaN
// (the reference's T**0.7 does for T < 0; T = 0 does not arise).
__device__ __forceinline__ double pow07(double T)
{
#ifndef CHAN_POW_HALLEY
    // y = T * x with x = T^-0.3, the root of x^10 T^3 = 1.  From the float seed
    // x0 (relative error ~3e-7), e = 1 - x0^10 T^3 and
    // x = x0 (1 - e)^(-1/10) = x0 (1 + e/10 + 0.055 e^2 + 0.0385 e^3 + ...):
    // the series to e^2 leaves ~1e-18; no division.
    const double x0 = (double)seed_exp2(-0.3f * seed_log2((float)T));
    const double t2 = T * T, t3 = t2 * T;
    const double x2 = x0 * x0, x4 = x2 * x2, x8 = x4 * x4, x10 = x8 * x2;
    const double e = fma(-x10, t3, 1.0);
    const double pe = fma(fma(0.0385, e, 0.055), e, 0.1);
    return T * fma(x0 * e, pe, x0);
#else
    const float tf = (float)T;
    double y = (double)seed_exp2(0.7f * seed_log2(tf));
    const double T2 = T * T, T4 = T2 * T2, a = (T4 * T2) * T;
    const double y2 = y * y, y4 = y2 * y2, y8 = y4 * y4, u = y8 * y2;
    const double num = fma(9.0, u, 11.0 * a);
    const double den = fma(11.0, u, 9.0 * a);
    return (y * num) * rcp_fast(den);
#endif
}

// primitives of one point from the conservative state (calcPrim, main_v1.9.f90:600-609)
__device__ __forceinline__ void prims_from_q(const KParams &P, const double q[5], double &u, double &v,
                                             double &w, double &T)
{
    const double r = rcp_fast(q[0]);
    u = q[1] * r;
    v = q[2] * r;
    w = q[3] * r;
    const double E = q[4] * r;
    // explicit FMAs: the same bits wherever a point's primitives are formed
    T = __fma_rn(-P.ggMh, __fma_rn(w, w, __fma_rn(v, v, u * u)), E);
}

// ---------------------------------------------------------------------------
// The fused stage kernel.
//
// A CTA owns a TI x TJ tile of interior (i,j) columns and marches a chunk of
// interior planes k = kb..ke.  Shared memory holds, for the tile plus a
// 2-point halo box ((TI+4) x (TJ+4)):
//   Q (5 vars)      of planes t, t+1, t+2   (3-slot ring; t+2 in flight)
//   prims u,v,w,T   of planes t, t+1        (2-slot ring)
//   mu, p           of planes t, t+1        (2-slot ring; mu only with float rings)
//   fD, gD          of plane t on the tile plus a 1-point halo
// Plane t-1 is kept where it is still read: each thread's own column (Q, u,
// v, w) in registers, and the halo points of the halo-flux lanes in a small
// shared array.  Each thread also keeps its own column's Q and w at t-2 and
// hD at t-1, t, t+1 in registers.
//
// The Q box of each plane arrives by one tiled bulk tensor copy (TMA) issued
// about two thirds of a plane ahead by one thread and completed on an mbarrier,
// so Q is read from DRAM once per stage with no per-thread load instructions;
// the halo re-reads of neighbouring CTAs come from L2.  Each staged box point is
// then converted to primitives once per CTA.  The stage whose input is stored in
// a wider type than the ring (the first stage of the mixed-precision path, double
// in, float rings) loads its boxes with per-thread loads instead.
//
// A plane takes two CTA barriers: after the box conversion (with which the
// inviscid x/y sums of the plane and the next own-column conversion share one
// straight-line block) and after the viscous fluxes.  None ends the plane, so
// warps that finish the update early go on into the next plane's loads and
// conversion while the others complete theirs.
//
// Types: QI / QO are the storage types of the stage's input and output state,
// R the type of the shared rings and of the flux arithmetic.  The plain FP64
// path is <double, double, double>.  The mixed-precision path stores the
// intermediate stage states in float and evaluates the fluxes in float; the
// primitive recovery (T from the total energy), the RK update against the
// double base state, the forcing and the blow-up test stay in double.
#ifndef CHAN_MINB
#define CHAN_MINB 2   // resident 256-thread CTAs per SM the register budget is sized for (FP64 rings)
#endif
#ifndef CHAN_MINB_F
#define CHAN_MINB_F 3 // the same with float rings (half the shared memory)
#endif

template <int TI, int TJ, typename R>
struct StageShape {
    static constexpr int BX = TI + 4, BY = TJ + 4, NB = BX * BY, NT = TI * TJ;
    // FP64 rings with 32-wide tiles: the own point's RK base arrives by a bulk
    // copy of the tile (tma_base); the room for it comes from forming p from
    // rho and T (no p ring) and exchanging fD along x by warp shuffles (a warp
    // is a row of the tile), which leaves only the two halo columns in sF.
#ifdef CHAN_TMA_BASE
    static constexpr bool tma_base = sizeof(R) == 8 && TI == 32;
#else
    static constexpr bool tma_base = false;
#endif
    static constexpr bool fx_shfl = tma_base;
    // where the own column of plane t+2 is read (measured per ring type: the FP64
    // kernel 7% faster reading its Q twice than holding it in registers, whose
    // spills it removes; the float kernels 2-3% faster loading it in phase C)
#if defined(CHAN_EARLY_T2)
    static constexpr bool late_t2 = false, late_qp2 = false;
#else
    static constexpr bool late_t2 = sizeof(R) == 4, late_qp2 = sizeof(R) == 8;
#endif
    static constexpr int NFX = fx_shfl ? 2 * TJ : TJ * (TI + 2), NGY = (TJ + 2) * TI;
    // float rings keep mu only and form p from rho and T where it is used;
    // FP64 rings keep (mu, p) unless the RK base takes the room
    static constexpr bool p_ring = sizeof(R) == 8 && !tma_base;
    static constexpr int MPW = p_ring ? 2 : 1;                       // words per box point in the (mu, p) ring
    // one Q slot: the 5-variable box of one plane, rounded up to 128 bytes
    // (the alignment of a bulk tensor copy's shared-memory destination)
    static constexpr size_t box_bytes = (size_t)5 * NB * sizeof(R);
    static constexpr size_t qslot_bytes = (box_bytes + 127) / 128 * 128;
    static constexpr int QSLOT = (int)(qslot_bytes / sizeof(R));     // slot stride in R elements
    static constexpr size_t q_bytes = 3 * qslot_bytes;
    static constexpr int pr_words = 2 * 4 * NB;
    static constexpr int mp_words = 2 * MPW * NB;
    static constexpr int fg_words = 4 * NFX + 4 * NGY;
    // float rings leave room to stage the RK base of every thread's own point
    // (double) by cp.async; the FP64 rings do not fit it beside two CTAs per SM
    static constexpr bool prefetch_base = sizeof(R) == 4;
    static constexpr bool base_slot = prefetch_base || tma_base;
    // the base slot is a bulk-copy destination: 128-byte aligned
    static constexpr size_t base_off = (q_bytes + sizeof(R) * (size_t)(pr_words + mp_words + fg_words) + 127) / 128 * 128;
    // plane t-1 values (u or v, and w) of the halo-flux lanes' points, by lane
    static constexpr int NHL = 32 + 2 * TI;
    static constexpr size_t hl_off = base_off + (base_slot ? sizeof(double) * 5 * (size_t)NT : 0);
    static constexpr size_t bar_off = (hl_off + sizeof(R) * 2 * (size_t)NHL + 7) / 8 * 8;
    static constexpr size_t bytes = bar_off + 4 * sizeof(unsigned long long) + 2 * sizeof(int);
    // resident CTAs per SM the register budget is sized for: 128 (FP64) or 80
    // (float) registers per thread at 256 threads, but never more CTAs than
    // the 228 KB of shared memory per SM holds (1 KB of it reserved per CTA)
    static constexpr int minb_regs = (sizeof(R) == 4 ? CHAN_MINB_F : CHAN_MINB) * 256 / NT;
    static constexpr int minb_smem = (int)(233472 / (bytes + 1024));
    static constexpr int minb = minb_regs < minb_smem ? minb_regs : minb_smem;
};

template <typename R>
__device__ __forceinline__ const FluxC<R> &fluxc(const KParams &P);
template <>
__device__ __forceinline__ const FluxC<double> &fluxc<double>(const KParams &P) { return P.cd; }
template <>
__device__ __forceinline__ const FluxC<float> &fluxc<float>(const KParams &P) { return P.cf; }

// per-k tables: 0 czh, 1 cz8, 2 cz12, 3 pez
template <typename R>
__device__ __forceinline__ R ktab(const KParams &P, int which, int k);
template <>
__device__ __forceinline__ double ktab<double>(const KParams &P, int which, int k)
{
    return which == 0 ? P.czh[k] : (which == 1 ? P.cz8[k] : (which == 2 ? P.cz12[k] : P.pez[k]));
}
template <>
__device__ __forceinline__ float ktab<float>(const KParams &P, int which, int k)
{
    return P.tabf[which * (P.n3 + 2) + k];
}

// mu = T^0.7 in the ring type: pow07 in double; exp2(0.7 log2 T) in float
template <typename R>
__device__ __forceinline__ R mu_of(double T);
template <>
__device__ __forceinline__ double mu_of<double>(double T) { return pow07(T); }
template <>
__device__ __forceinline__ float mu_of<float>(double T)
{
    // the hardware log2 and exp2 approximations (relative error about 2^-21, well
    // inside the float path's own rounding); the library log2f/exp2f cost 2.5% of
    // the float stage kernel (CHAN_LIBM_MU_F)
#ifndef CHAN_LIBM_MU_F
    return seed_exp2(0.7f * seed_log2((float)T));
#else
    return exp2f(0.7f * log2f((float)T));
#endif
}

// a load of state written earlier in the same launch by other CTAs (the
// persistent ensemble kernel) must not use the read-only path
template <bool COHERENT, typename T>
__device__ __forceinline__ double ldq_c(const T *p) { return COHERENT ? (double)*p : (double)__ldg(p); }

// 8-byte asynchronous global->shared copy (no register staging)
__device__ __forceinline__ void cp_async8(double *dst, const double *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---- tiled bulk tensor copies into this CTA's shared memory, with mbarriers
__device__ __forceinline__ unsigned smem_u32addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init_one(unsigned long long *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32addr(bar)) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// order the CTA's earlier generic-proxy accesses of shared memory (made
// visible to this thread by a CTA barrier) before its later async-proxy writes
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// the 4-D box at (x, y, z, w) of the tensor map into dst; bytes = box size.
// No multicast: the box lands in this CTA's shared memory only.
__device__ __forceinline__ void tma_load_box(void *dst, const CUtensorMap *map, int x, int y, int z, int w,
                                             unsigned long long *bar, unsigned bytes)
{
    const unsigned b = smem_u32addr(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_u32addr(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(b)
        : "memory");
}

__device__ __forceinline__ bool mbar_try(unsigned a, unsigned parity)
{
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// wait for phase `parity` of the barrier; false when about a second passed
// without it (the caller records the error and stops)
constexpr unsigned long long kCopyWaitNs = 1000000000ull;
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity)
{
    const unsigned a = smem_u32addr(bar);
    if (mbar_try(a, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try(a, parity))
        if (global_ns() - t0 > kCopyWaitNs) return false;
    return true;
}

// One CTA's work of the stage kernel on tile (bx, by) and k-chunk bz, for
// thread (tx, ty).  BUOYM: 0 no buoyancy term, 1 with it, 2 as P.buoy_on
// says.  PERSIST: called from the persistent ensemble kernel, where the state
// was written earlier in the same launch: coherent loads instead of the
// read-only path, and a proxy fence before the first box copy.
template <int TI, int TJ, typename QI, typename QO, typename R, int BUOYM, bool PERSIST>
__device__ __forceinline__ void stage_body(const KParams &P, const CUtensorMap *tmq, const CUtensorMap *tmb, int bx,
                                           int by, int bz, int tx, int ty, unsigned char *smem_raw)
{
    using S = StageShape<TI, TJ, R>;
    using Slot = SlotT<R>;
    constexpr bool late_t2 = S::late_t2, late_qp2 = S::late_qp2;
    constexpr int BX = S::BX, BY = S::BY, NB = S::NB, NT = S::NT, MPW = S::MPW, QSLOT = S::QSLOT;
    // boxes by bulk tensor copy when the input is stored in the ring type
#ifdef CHAN_NO_TMA
    constexpr bool TMA = false;   // measurement variant: per-thread box loads into the same ring
#else
    constexpr bool TMA = std::is_same<QI, R>::value;
#endif
    static_assert(2 * TJ <= 32 && 32 + 2 * TI <= NT, "halo-flux lane layout needs 2*TJ <= 32 and 32+2*TI <= TI*TJ");
    R *sQ = reinterpret_cast<R *>(smem_raw);                       // [3 slots][5][NB]
    R *sPr = reinterpret_cast<R *>(smem_raw + S::q_bytes);         // [2][4][NB] u,v,w,T
    R *sMP = sPr + S::pr_words;                                    // [2][MPW][NB] mu (, p)
    R *sF = sMP + S::mp_words;                                     // [4][TJ][TI+2]
    R *sG = sF + 4 * S::NFX;                                       // [4][TJ+2][TI]
    double *sQB = reinterpret_cast<double *>(smem_raw + S::base_off);   // [5][NT] (float rings only)
    R *sH = reinterpret_cast<R *>(smem_raw + S::hl_off);                // [2][NHL]
    // (the 8-byte rounding is a no-op: bar_off is a multiple of 8)
    unsigned long long *bar = reinterpret_cast<unsigned long long *>(reinterpret_cast<size_t>(smem_raw + S::bar_off) & ~(size_t)7);   // [3]
    int *sflag = reinterpret_cast<int *>(bar + 4);   // [0] the CTA leaves at once, [1] slots with a copy in flight
    const FluxC<R> &C = fluxc<R>(P);
    // the state pointers are read from the parameter space at each use: held
    // in registers across the kernel they cost spills
    auto qin = [&]() { return static_cast<const QI *>(P.qin); };
    auto qout = [&]() { return static_cast<QO *>(P.qout); };

    const bool buoy = BUOYM == 2 ? P.buoy_on != 0 : BUOYM == 1;
    const int tid = ty * TI + tx;
    if (tid == 0) {
        sflag[0] = frozen(P.status, kstep(P)) ? 1 : 0;
        sflag[1] = 0;
        // state written by other CTAs of this launch, read next by box copies
        if (PERSIST) asm volatile("fence.proxy.async.global;" ::: "memory");
        // a bulk copy needs a 128-byte aligned destination
        if (TMA && (smem_u32addr(smem_raw) & 127u)) {
            sflag[0] = 1;
            atomicExch(&P.status->stall, 2);
        }
        if (TMA || S::tma_base) {
            for (int s = 0; s < 4; s++) mbar_init_one(&bar[s]);
            fence_mbar_init();
        }
    }
    __syncthreads();
    if (sflag[0]) return;

    const int i0 = 2 + bx * TI, j0 = 2 + by * TJ;
    const int kb = 2 + bz * P.kchunk;
    const int ke = min(kb + P.kchunk - 1, P.n3 - 1);
    if (kb > ke) return;
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3;
    const int i = i0 + tx, j = j0 + ty;
    const bool col_ok = (i <= n1) && (j <= n2);
    const bool out_ok = (i <= n1 - 1) && (j <= n2 - 1);
    const int bc = (ty + 2) * BX + (tx + 2);
    const long long vol = P.vol, plane = P.plane;
    const long long colo = (long long)j * P.px + i;

    // ring slots by role, rotated once per plane: Q slots (indices 0..2) of
    // planes t, t+1, t+2; prims offsets of t, t+1; (mu,p) offsets of t, t+1
    int iZ = 1, iP = 2, iN = 0;
    int pZ = 0, pP = 4 * NB, mZ = 0, mP = MPW * NB;
    unsigned ph = 0u;   // parity of the next wait, per Q slot
    auto slot = [&](int o) -> Slot {
        return Slot{sPr + o, sPr + o + NB, sPr + o + 2 * NB, sPr + o + 3 * NB};
    };
    auto smu = [&](int o) { return sMP + o; };
    auto sq = [&](int s, int v) { return sQ + s * QSLOT + v * NB; };
    // what the flux helpers read the pressure from (pres_at): the p slot of
    // the (mu,p) ring at mo, or the density of the Q slot s
    auto spr = [&](int mo, int s) { return S::p_ring ? sMP + mo + NB : sq(s, 0); };

    // plane m's Q box into Q slot s (one thread; bulk tensor copy)
    auto issue = [&](int m, int s) {
        if (TMA && tid == 0) {
            fence_proxy_async_smem();
            tma_load_box(sq(s, 0), tmq, i0 - 2, j0 - 2, m, 0, &bar[s], (unsigned)S::box_bytes);
            sflag[1] |= 1 << s;
        }
    };
    // wait for Q slot s; false if the copy did not complete in time
    auto wait_slot = [&](int s) -> bool {
        if (s < 3 ? !TMA : !S::tma_base) return true;
        const bool ok = mbar_wait_bounded(&bar[s], (ph >> s) & 1u);
        ph ^= 1u << s;
        if (ok && tid == 0) sflag[1] &= ~(1 << s);
        return ok;
    };
    // after a timed-out copy: record it, give every copy still in flight one
    // more bounded wait (so that none lands after the CTA has left), leave
    auto give_up = [&]() {
        if (tid == 0) {
            atomicExch(&P.status->stall, 1);
            for (int s = 0; s < 4; s++)
                if (sflag[1] & (1 << s)) mbar_wait_bounded(&bar[s], (ph >> s) & 1u);
        }
    };
    // the tile's RK base of plane m into the base slot (barrier 3)
    auto issue_base = [&](int m) {
        if (S::tma_base && tid == 0) {
            fence_proxy_async_smem();
            tma_load_box(sQB, tmb, i0, j0, m, 0, &bar[3], (unsigned)(sizeof(double) * 5 * NT));
            sflag[1] |= 1 << 3;
        }
    };

    // box points this thread converts: the same columns for every plane
    // lp: box index | 0x10000 if the point is in R1 (tile plus a 1-point cross
    // halo, where mu and p are needed); -1 if outside the array.  lo: column offset.
    constexpr int NL = (NB + NT - 1) / NT;
    int lp[NL];
    int lo[NL];
#pragma unroll
    for (int l = 0; l < NL; l++) {
        const int p = tid + l * NT;
        const int bj = p / BX, bi = p - bj * BX;
        const int gi = i0 - 2 + bi, gj = j0 - 2 + bj;
        const bool ok = p < NB && gi <= n1 + 1 && gj <= n2 + 1;
        const bool r1 = (bi >= 1 && bi <= BX - 2 && bj >= 2 && bj <= BY - 3) ||
                        (bi >= 2 && bi <= BX - 3 && bj >= 1 && bj <= BY - 2);
        lp[l] = ok ? (p | (r1 ? 0x10000 : 0)) : -1;
        lo[l] = gj * P.px + gi;
    }

    // The inviscid x and y flux derivatives of plane t (F1 + G1) need only plane
    // t's Q box and u, v, which the previous plane converted: they are formed in
    // phase A, in the same straight-line block as the conversion of plane t+1's
    // box, whose dependency chains (reciprocal, power) they fill (1.7% of the
    // FP64 stage time, 2.4% of the float one, against forming them in phase E;
    // in phase C, beside the viscous fluxes, they were 2.8% slower than in E).
    // CHAN_XY_IN_E keeps them in phase E, for measurement.
#ifdef CHAN_XY_IN_E
    constexpr bool xy_a = false;
#else
    constexpr bool xy_a = true;
#endif
    R Fxy[5] = {0, 0, 0, 0, 0};
    auto inv_xy = [&]() {
        const R mu0 = smu(mZ)[bc];
        const R *U = sPr + pZ, *V = sPr + pZ + NB;
        const bool qx = (C.pex * fabs(sq(iZ, 1)[bc])) > C.PexVal * mu0;
        const bool qy = (C.pey * fabs(sq(iZ, 2)[bc])) > C.PeyVal * mu0;
        R wx[5], wy[5];
        inv_weights(U[bc - 2], U[bc - 1], U[bc], U[bc + 1], U[bc + 2], qx, C.sx8, C.sx12, wx);
        inv_weights(V[bc - 2 * BX], V[bc - BX], V[bc], V[bc + BX], V[bc + 2 * BX], qy, C.sy8, C.sy12, wy);
#pragma unroll
        for (int c = 0; c < 5; c++) {
            const R *Q = sq(iZ, c);
            Fxy[c] = wsum(wx, Q[bc - 2], Q[bc - 1], Q[bc], Q[bc + 1], Q[bc + 2]) +
                     wsum(wy, Q[bc - 2 * BX], Q[bc - BX], Q[bc], Q[bc + BX], Q[bc + 2 * BX]);
        }
    };

    // primitives (and mu, p on R1) of plane m over the box, from its Q box in
    // slot s (with per-thread loads, Q is first loaded into the slot).  A wall
    // plane's box holds, at periodic duplicates and ghosts, the values of their
    // image points: the viscous fluxes next to a wall read the wall only there,
    // and the reference's flux at a duplicate column or row is the exchanged
    // flux of its image (whose wall values may differ from the duplicate's own
    // under a non-periodic wall BC).  hD on a wall plane reads the wall's own
    // values from memory instead (hflux_wall).
    auto no_extra = []() {};
    // FP64 rings: mu (and p) formed and stored at every box point, not only on R1,
    // where they are read (the other cells of the slot are never read): the
    // conversion's block then has no branch on R1, and the 1.31 -> 1.69 powers per
    // output cost less than the divergent branch did (2.9% of the FP64 stage time;
    // the float kernels, whose float mu is cheap, are 0.9% slower with it).
    // CHAN_MU_R1 keeps the branch, for measurement.
#ifdef CHAN_MU_R1
    constexpr bool mu_all = false;
#else
    constexpr bool mu_all = sizeof(R) == 8;
#endif
    auto convert = [&](int m, int s, int po, int mo, bool with_xy, auto &&extra) {
        const Slot sl = slot(po);
        R *MU = smu(mo), *PR = sMP + mo + NB;
        const bool wall = (m == 1 || m == n3);
        const double *W = P.wp + (size_t)(m == 1 ? 0 : 8) * plane;
        auto one = [&](int l, bool wall_plane) {
            if (lp[l] < 0) return;
            const int p = lp[l] & 0xffff;
            const bool r1 = (lp[l] & 0x10000) != 0;
            double q[5];
            if (!TMA) {
                const long long off = (long long)m * plane + lo[l];
#pragma unroll
                for (int v = 0; v < 5; v++) {
                    q[v] = ldq_c<PERSIST>(qin() + v * vol + off);
                    sq(s, v)[p] = (R)q[v];
                }
            }
            double u, vv, w, T, pr;
            R mu;
            if (wall_plane) {
                const int bj = p / BX, bi = p - bj * BX;
                const long long wo = (long long)wrap_idx(j0 - 2 + bj, n2) * P.px + wrap_idx(i0 - 2 + bi, n1);
                u = W[1 * plane + wo];
                vv = W[2 * plane + wo];
                w = W[3 * plane + wo];
                T = W[5 * plane + wo];
                pr = W[6 * plane + wo];
                mu = (R)W[7 * plane + wo];
            } else {
                if (TMA) {
#pragma unroll
                    for (int v = 0; v < 5; v++) q[v] = (double)sq(s, v)[p];
                }
                prims_from_q(P, q, u, vv, w, T);
                pr = (q[0] * T) * P.inv_gM2;
                mu = mu_all ? mu_of<R>(T) : (r1 ? mu_of<R>(T) : R(0));
            }
            ((R *)sl.U)[p] = (R)u;
            ((R *)sl.V)[p] = (R)vv;
            ((R *)sl.W)[p] = (R)w;
            ((R *)sl.T)[p] = (R)T;
            if (mu_all || r1) {
                MU[p] = mu;
                if (S::p_ring) PR[p] = (R)pr;
            }
        };
        // the wall test taken once per plane, so that each loop's body is
        // straight-line code (2.6% of the FP64 stage time against one loop with the
        // test inside); the per-thread box loads one box point at a time, with fewer
        // loads in flight (0.4% of the mean float stage time)
        auto loop = [&](bool wall_plane) {
            if (!TMA) {
#pragma unroll 1
                for (int l = 0; l < NL; l++) one(l, wall_plane);
            } else {
#pragma unroll
                for (int l = 0; l < NL; l++) one(l, wall_plane);
            }
            if (xy_a && with_xy) inv_xy();
            extra();
        };
        if (wall) loop(true);
        else loop(false);
    };

    // own-column Q and u,v,w,T of plane m read straight from memory
    auto center = [&](int m, double q[5], double &u, double &v, double &w, double &T) {
        const long long off = (long long)m * plane + colo;
#pragma unroll
        for (int c = 0; c < 5; c++) q[c] = ldq_c<PERSIST>(qin() + c * vol + off);
        if (m == 1 || m == n3) {
            const double *W = P.wp + (size_t)(m == 1 ? 0 : 8) * plane + colo;
            u = W[1 * plane]; v = W[2 * plane]; w = W[3 * plane]; T = W[5 * plane];
        } else {
            prims_from_q(P, q, u, v, w, T);
        }
    };

    // hD at the own column of interior plane m (prims at po, (mu,p) at mo, Q
    // slot s); dz from (m-1, m+1) values
    auto hflux = [&](int m, int po, int mo, int s, R um, R vm, R wm, R Tm, R up, R vp, R wp_, R Tp, R h[4]) {
        const Slot sl = slot(po);
        const R sc = ktab<R>(P, 0, m);
        visc_fz<BX>(C, sl, smu(mo)[bc], pres_at<R, S::p_ring>(C, sl, spr(mo, s), bc), bc, (up - um) * sc, (vp - vm) * sc,
                    (wp_ - wm) * sc, (Tp - Tm) * sc, h);
    };
    // hD at the own column of wall plane m, from the wall's own values in
    // memory, in double; one-sided dz against the interior neighbour values
    // (ui..Ti): (q(2)-q(1))/dz1 at the bottom, (q(nP3)-q(nP3-1))/dzN at the
    // top.  The pressure is the pressure-BC state.
    auto hflux_wall = [&](int m, double ui, double vi, double wi, double Ti, double h[4]) {
        const double *W = P.wp + (size_t)(m == 1 ? 0 : 8) * plane + colo;
        const long long px = P.px;
        const double u0 = W[plane], v0 = W[2 * plane], w0 = W[3 * plane], T0 = W[5 * plane];
        const double sc = m == 1 ? P.inv_dz1 : P.inv_dzN;
        const double ux = (W[plane + 1] - W[plane - 1]) * P.hdx;
        const double vy = (W[2 * plane + px] - W[2 * plane - px]) * P.hdy;
        const double wx = (W[3 * plane + 1] - W[3 * plane - 1]) * P.hdx;
        const double wy = (W[3 * plane + px] - W[3 * plane - px]) * P.hdy;
        const double uz = (m == 1 ? ui - u0 : u0 - ui) * sc, vz = (m == 1 ? vi - v0 : v0 - vi) * sc;
        const double wz = (m == 1 ? wi - w0 : w0 - wi) * sc, Tz = (m == 1 ? Ti - T0 : T0 - Ti) * sc;
        visc_fz_vals(P.cd, ux, vy, wx, wy, u0, v0, w0, W[7 * plane], W[6 * plane], uz, vz, wz, Tz, h);
    };

    // halo-flux lanes: fD of the two x-halo columns on lanes 0..2TJ-1 of warp
    // 0, gD of the two y-halo rows on lanes 32..32+2TI-1.  Each owns one halo
    // point for the whole march and keeps that point's plane t-1 values (u or
    // v, and w) in sH[.][tid].  hbox: the point's box index.
    const bool hx_lane = tid < 2 * TJ;
    const bool hy_lane = tid >= 32 && tid < 32 + 2 * TI;
    auto hbox = [&]() -> int {
        if (hx_lane) {
            const int side = tid / TJ, r = tid - side * TJ;
            return (r + 2) * BX + (side ? TI + 2 : 1);
        }
        const int h = tid - 32, side = h / TI, cc = h - side * TI;
        return (side ? TJ + 2 : 1) * BX + cc + 2;
    };
    // the halo lane's values (u or v, w) in ring slot sl, kept as plane t-1
    auto keep_halo = [&](const Slot &sl) {
        if (hx_lane || hy_lane) {
            const int b = hbox();
            sH[tid] = hx_lane ? sl.U[b] : sl.V[b];
            sH[S::NHL + tid] = sl.W[b];
        }
    };

    // ---------------- prologue: planes kb-1 (Q slot 0, prims at pP) and kb
    // (Q slot 1, prims at pZ); hD(kb-1), hD(kb); plane kb+1 starts its way in
    issue(kb - 1, 0);
    issue(kb, 1);
    issue(kb + 1, 2);   // kb+1 <= ke+1 <= nP3
    bool bad = !wait_slot(0);
    convert(kb - 1, 0, pP, mP, false, no_extra);
    bad = !wait_slot(1) || bad;
    convert(kb, 1, pZ, mZ, false, no_extra);
    if (__syncthreads_or(bad)) { give_up(); return; }

    R qm2[5] = {0, 0, 0, 0, 0}, qm1[5], hm1[4] = {0, 0, 0, 0}, h0[4] = {0, 0, 0, 0};
    R wm2 = R(0), um1 = R(0), vm1 = R(0), wm1 = R(0);   // own column: w at t-2; u, v, w at t-1
    {
        const Slot sA = slot(pP), sB = slot(pZ);
        if (col_ok) {
            // hD(kb-1)
            if (kb - 1 == 1) {
                double h[4];
                hflux_wall(1, sB.U[bc], sB.V[bc], sB.W[bc], sB.T[bc], h);
#pragma unroll
                for (int c = 0; c < 4; c++) hm1[c] = (R)h[c];
            } else {
                double q[5], u, v, w, T;
                center(kb - 2, q, u, v, w, T);
                hflux(kb - 1, pP, mP, 0, (R)u, (R)v, (R)w, (R)T, sB.U[bc], sB.V[bc], sB.W[bc], sB.T[bc], hm1);
            }
            // hD(kb)
            {
                double q[5], u, v, w, T;
                center(kb + 1, q, u, v, w, T);
                hflux(kb, pZ, mZ, 1, sA.U[bc], sA.V[bc], sA.W[bc], sA.T[bc], (R)u, (R)v, (R)w, (R)T, h0);
            }
            if (kb - 2 >= 1) {
                double q[5], u, v, w, T;
                center(kb - 2, q, u, v, w, T);
#pragma unroll
                for (int c = 0; c < 5; c++) qm2[c] = (R)q[c];
                wm2 = (R)w;
            }
            // the last chunk stages hD of the top wall plane for its last plane
            if (ke == n3 - 1) {
                double q[5], u, v, w, T, h[4];
                center(n3 - 1, q, u, v, w, T);
                hflux_wall(n3, u, v, w, T, h);
#pragma unroll
                for (int c = 0; c < 4; c++) P.hwt[c * plane + colo] = h[c];
            }
#pragma unroll
            for (int c = 0; c < 5; c++) qm1[c] = sq(0, c)[bc];
            um1 = sA.U[bc]; vm1 = sA.V[bc]; wm1 = sA.W[bc];
        } else {
#pragma unroll
            for (int c = 0; c < 5; c++) qm1[c] = R(0);
        }
        keep_halo(sA);
    }
    __syncthreads();

    for (int t = kb; t <= ke; t++) {
        // ---------- A: own column of t+2; (float rings: the own point's RK base
        // starts its way into shared memory); plane t+1's box is converted, beside
        // the inviscid x/y sums of plane t; after the barrier, plane t+2's box
        // starts its way in (converted at the next plane)
        // No barrier ends the plane (neb), so a warp that has finished plane t's
        // update goes on to plane t+1's loads, box wait and conversion while others
        // still run phase E.  What makes that safe: plane t+2's box goes into the
        // slot of plane t-1 only after phase A's barrier, which every thread passes
        // after its phase-E reads of that slot; and what phases E and F read of
        // plane t's primitive and (mu, p) slots, which the next plane's conversion
        // overwrites, is read before barrier C.  FP64 stage time 3.5% lower together
        // with the split own-column conversion below (alone 1% higher); float 1%
        // lower.  CHAN_END_BAR restores the barrier, for measurement.
#ifndef CHAN_END_BAR
        constexpr bool neb = !S::tma_base;
#else
        constexpr bool neb = false;
#endif
        if (t < ke && !neb) issue(t + 2, iN);
        const bool need_base = P.rk_mode != 0;
        if (S::tma_base && need_base) issue_base(t);
        if (S::prefetch_base) {
            if (P.rk_mode != 0 && out_ok) {
                const double *src = P.qbase + (long long)t * plane + colo;
#pragma unroll
                for (int c = 0; c < 5; c++) cp_async8(sQB + c * NT + tid, src + c * vol);
            }
            cp_async_commit();
        }
#ifndef CHAN_NO_PREFETCH_BASE_L1
        // the own point's RK base into L1 now; the update reads it at the end of
        // the plane (2.7% of the FP64 stage time against loading it there cold)
        if (!S::prefetch_base && !S::tma_base && P.rk_mode != 0 && out_ok) {
            const double *src = P.qbase + (long long)t * plane + colo;
#pragma unroll
            for (int c = 0; c < 5; c++) asm volatile("prefetch.global.L1 [%0];" ::"l"(src + c * vol));
        }
#endif
        // FP64: plane t+3's own column into L1 a plane before it is loaded (1.8% of the
        // FP64 stage time; the float kernels, which load plane t+2 in phase C, are
        // slower with it)
        if (sizeof(R) == 8 && col_ok && t + 3 <= n3) {
            const QI *src = qin() + (long long)(t + 3) * plane + colo;
#pragma unroll
            for (int c = 0; c < 5; c++) asm volatile("prefetch.global.L1 [%0];" ::"l"(src + c * vol));
        }
        R qp2[5] = {0, 0, 0, 0, 0}, up2 = 0, vp2 = 0, wp2 = 0, Tp2 = 0;
        // FP64: plane t+2's own column is loaded before the box wait and converted
        // after it, in the straight-line block of the box conversion (1.9% of the
        // stage time alone, 3.5% with neb); CHAN_T2_JOINED converts it at its load
#ifndef CHAN_T2_JOINED
        constexpr bool t2_split = !late_t2;
#else
        constexpr bool t2_split = false;
#endif
        const bool own2 = col_ok && t + 2 < n3;   // plane t+2's own column is an interior one
        double cq[5] = {0, 0, 0, 0, 0};
        // plane t+2's own column: the float kernels prefetch it into L1 here and
        // load and convert it in phase C, where its values start to be used; the
        // FP64 kernel loads and converts it here but reads its Q again in phase E
        // (an L1 hit) instead of keeping it in registers across the plane
        if (late_t2) {
            if (col_ok && t + 2 <= n3) {
                const QI *src = qin() + (long long)(t + 2) * plane + colo;
#pragma unroll
                for (int c = 0; c < 5; c++) asm volatile("prefetch.global.L1 [%0];" ::"l"(src + c * vol));
            }
        } else if (t2_split && own2) {
            // interior plane t+2: its own column's Q now, its primitives after the box wait
            const long long off = (long long)(t + 2) * plane + colo;
#pragma unroll
            for (int c = 0; c < 5; c++) cq[c] = ldq_c<PERSIST>(qin() + c * vol + off);
        } else if (col_ok && t + 2 <= n3) {
            double q[5], u, v, w, T;
            center(t + 2, q, u, v, w, T);
            if (!late_qp2) {
#pragma unroll
                for (int c = 0; c < 5; c++) qp2[c] = (R)q[c];
            }
            up2 = (R)u; vp2 = (R)v; wp2 = (R)w; Tp2 = (R)T;
        }
        // the primitives of plane t+2's own column formed in the same straight-line
        // block as the box conversion (selects keep the other cases' values)
        auto t2_prims = [&]() {
            if (t2_split) {
                double u, v, w, T;
                prims_from_q(P, cq, u, v, w, T);
                up2 = own2 ? (R)u : up2;
                vp2 = own2 ? (R)v : vp2;
                wp2 = own2 ? (R)w : wp2;
                Tp2 = own2 ? (R)T : Tp2;
                if (!late_qp2) {
#pragma unroll
                    for (int c = 0; c < 5; c++) qp2[c] = own2 ? (R)cq[c] : qp2[c];
                }
            }
        };
        bad = !wait_slot(iP);
        convert(t + 1, iP, pP, mP, true, t2_prims);
        if (__syncthreads_or(bad)) { give_up(); return; }
        if (t < ke && neb) issue(t + 2, iN);

        // ---------- C: viscous flux vectors
        const Slot s0 = slot(pZ), sp = slot(pP);
        R hp1[4] = {0, 0, 0, 0};
        R fown[4] = {0, 0, 0, 0};   // fD at the own column (exchanged by shuffles when fx_shfl)
        {
            const R czt = ktab<R>(P, 0, t);
            const R *MU = smu(mZ), *PR = spr(mZ, iZ);
            if (col_ok) {
                if (late_t2 && t + 2 <= n3) {
                    double q[5], u, v, w, T;
                    center(t + 2, q, u, v, w, T);
#pragma unroll
                    for (int c = 0; c < 5; c++) qp2[c] = (R)q[c];
                    up2 = (R)u; vp2 = (R)v; wp2 = (R)w; Tp2 = (R)T;
                }
                // FP64 rings: hD(t+1) on every plane (on the top wall plane it reads the
                // wall's valid ring values and is not used), so that it shares one
                // straight-line block with fD and gD (0.9% of the FP64 stage time; the
                // float kernels keep the uniform branch, 0.2% faster).  CHAN_HFLUX_GUARD
                // keeps the branch in the FP64 kernel too, for measurement.
#ifdef CHAN_HFLUX_GUARD
                constexpr bool hflux_all = false;
#else
                constexpr bool hflux_all = sizeof(R) == 8;
#endif
                if (hflux_all) {
                    R h[4];
                    hflux(t + 1, pP, mP, iP, s0.U[bc], s0.V[bc], s0.W[bc], s0.T[bc], up2, vp2, wp2, Tp2, h);
                    const bool hok = t + 1 != n3;
#pragma unroll
                    for (int c = 0; c < 4; c++) hp1[c] = hok ? h[c] : R(0);
                } else if (t + 1 != n3) {
                    hflux(t + 1, pP, mP, iP, s0.U[bc], s0.V[bc], s0.W[bc], s0.T[bc], up2, vp2, wp2, Tp2, hp1);
                }
                R g[4];
                visc_fxy<BX, R, S::p_ring>(C, s0, um1, vm1, wm1, sp, MU, PR, bc, czt, fown, g);
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    if (!S::fx_shfl) sF[(c * TJ + ty) * (TI + 2) + tx + 1] = fown[c];
                    sG[(c * (TJ + 2) + ty + 1) * TI + tx] = g[c];
                }
            }
            if (hx_lane) {
                const int side = tid / TJ, r = tid - side * TJ;
                const int ci = side ? i0 + TI : i0 - 1, cj = j0 + r;
                if (ci <= n1 && cj <= n2) {
                    R f[4];
                    visc_fx<BX, R, S::p_ring>(C, s0, sH[tid], sH[S::NHL + tid], sp, MU, PR,
                                              (r + 2) * BX + (side ? TI + 2 : 1), czt, f);
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        if (S::fx_shfl) sF[c * S::NFX + r * 2 + side] = f[c];
                        else sF[c * S::NFX + r * (TI + 2) + (side ? TI + 1 : 0)] = f[c];
                    }
                }
            } else if (hy_lane) {
                const int h = tid - 32, side = h / TI, cc = h - side * TI;
                const int ci = i0 + cc, cj = side ? j0 + TJ : j0 - 1;
                if (ci <= n1 && cj <= n2) {
                    R g[4];
                    visc_fy<BX, R, S::p_ring>(C, s0, sH[tid], sH[S::NHL + tid], sp, MU, PR,
                                              (side ? TJ + 2 : 1) * BX + cc + 2, czt, g);
#pragma unroll
                    for (int c = 0; c < 4; c++) sG[c * S::NGY + (side ? TJ + 1 : 0) * TI + cc] = g[c];
                }
            }
        }
        // without the end-of-plane barrier, the next plane's conversion overwrites
        // plane t's primitive and (mu, p) slots while this plane's phase E may still
        // run: what phases E and F read of them is read here, before barrier C
        R w0n = R(0), mu0n = R(0), T0n = R(0);
        if (neb) {
            um1 = s0.U[bc]; vm1 = s0.V[bc];   // plane t-1's u, v are not read after phase C
            w0n = s0.W[bc];
            mu0n = smu(mZ)[bc];
            if (buoy) T0n = s0.T[bc];
            keep_halo(s0);
        }
        if (S::tma_base && need_base) {
            bad = !wait_slot(3);
            if (__syncthreads_or(bad)) { give_up(); return; }
        } else {
            __syncthreads();
        }

        // ---------- E: fluxes, source, RK update
        // fD at the x neighbours: lanes tx+-1 of the row's warp, the halo columns
        // at the row's ends (every lane takes part in the shuffles)
        R fxp[4], fxm[4];
        if (S::fx_shfl) {
#pragma unroll
            for (int c = 0; c < 4; c++) {
                fxp[c] = __shfl_down_sync(0xffffffffu, fown[c], 1);
                fxm[c] = __shfl_up_sync(0xffffffffu, fown[c], 1);
                if (tx == TI - 1) fxp[c] = sF[c * S::NFX + ty * 2 + 1];
                if (tx == 0) fxm[c] = sF[c * S::NFX + ty * 2 + 0];
            }
        }
        R q0[5];
#pragma unroll
        for (int c = 0; c < 5; c++) q0[c] = sq(iZ, c)[bc];
        if (out_ok) {
#ifdef CHAN_EARLY_BASE
            // the RK base of the own point, loaded before the flux sums so that
            // its latency overlaps them (FP64 rings)
            double qbe[5] = {0, 0, 0, 0, 0};
            if (!S::prefetch_base && P.rk_mode != 0) {
                const long long off = (long long)t * plane + colo;
#pragma unroll
                for (int c = 0; c < 5; c++) qbe[c] = ldq_c<PERSIST>(P.qbase + c * vol + off);
            }
#endif
            R Fs[5];   // sum of the flux derivatives
            const R mu0 = neb ? mu0n : smu(mZ)[bc];
            if (xy_a) {
                // (F1 + G1) from phase A, then the viscous x and y terms
                Fs[0] = Fxy[0];
#pragma unroll
                for (int c = 1; c < 5; c++) {
                    R F2;
                    if (S::fx_shfl) {
                        F2 = (fxp[c - 1] - fxm[c - 1]) * C.hdx;
                    } else {
                        const int r = (c - 1) * TJ + ty;
                        F2 = (sF[r * (TI + 2) + tx + 2] - sF[r * (TI + 2) + tx]) * C.hdx;
                    }
                    const R G2 = (sG[((c - 1) * (TJ + 2) + ty + 2) * TI + tx] -
                                  sG[((c - 1) * (TJ + 2) + ty) * TI + tx]) * C.hdy;
                    Fs[c] = (Fxy[c] + F2) + G2;
                }
            }
            // x
            if (!xy_a) {
                const R *U = s0.U;
                const bool qk = (C.pex * fabs(q0[1])) > C.PexVal * mu0;
                R w[5];
                inv_weights(U[bc - 2], U[bc - 1], U[bc], U[bc + 1], U[bc + 2], qk, C.sx8, C.sx12, w);
                R F1[5];
#pragma unroll
                for (int c = 0; c < 5; c++) {
                    const R *Q = sq(iZ, c);
                    F1[c] = wsum(w, Q[bc - 2], Q[bc - 1], Q[bc], Q[bc + 1], Q[bc + 2]);
                }
                Fs[0] = F1[0];  // F2 of continuity is zero
#pragma unroll
                for (int c = 1; c < 5; c++) {
                    R F2;
                    if (S::fx_shfl) {
                        F2 = (fxp[c - 1] - fxm[c - 1]) * C.hdx;
                    } else {
                        const int r = (c - 1) * TJ + ty;
                        F2 = (sF[r * (TI + 2) + tx + 2] - sF[r * (TI + 2) + tx]) * C.hdx;
                    }
                    Fs[c] = F1[c] + F2;
                }
            }
            // y
            if (!xy_a) {
                const R *V = s0.V;
                const bool qk = (C.pey * fabs(q0[2])) > C.PeyVal * mu0;
                R w[5];
                inv_weights(V[bc - 2 * BX], V[bc - BX], V[bc], V[bc + BX], V[bc + 2 * BX], qk, C.sy8, C.sy12, w);
                R G1[5];
#pragma unroll
                for (int c = 0; c < 5; c++) {
                    const R *Q = sq(iZ, c);
                    G1[c] = wsum(w, Q[bc - 2 * BX], Q[bc - BX], Q[bc], Q[bc + BX], Q[bc + 2 * BX]);
                }
                Fs[0] = Fs[0] + G1[0];
#pragma unroll
                for (int c = 1; c < 5; c++) {
                    const R G2 = (sG[((c - 1) * (TJ + 2) + ty + 2) * TI + tx] -
                                  sG[((c - 1) * (TJ + 2) + ty) * TI + tx]) * C.hdy;
                    Fs[c] = (Fs[c] + G1[c]) + G2;
                }
            }
            // z
            {
                const R w0 = neb ? w0n : s0.W[bc], wp1 = sp.W[bc];
                R w[5];
                // FP64 rings: the second-order weights of the planes next to the walls
                // and the hybrid ones both formed and selected by the (uniform) plane
                // test, so that the update's block has no branch (0.7% of the FP64 stage
                // time); CHAN_ZW_BRANCH keeps the branch, for measurement
#ifdef CHAN_ZW_BRANCH
                constexpr bool zw_sel = false;
#else
                constexpr bool zw_sel = sizeof(R) == 8;
#endif
                if (zw_sel) {
                    // both weight sets, selected by the (uniform) plane test: no branch
                    // in the update's block (the tables hold nP3+2 entries, so the
                    // interior set's reads stay in range on every plane)
                    const bool near = t < 3 || t > n3 - 2;
                    const R c2 = ktab<R>(P, 0, t);
                    const bool qk = (ktab<R>(P, 3, t) * fabs(q0[3])) > C.pez_val * mu0;
                    R wi[5];
                    inv_weights(wm2, wm1, w0, wp1, wp2, qk, ktab<R>(P, 1, t), ktab<R>(P, 2, t), wi);
                    w[0] = near ? R(0) : wi[0];
                    w[1] = near ? -(wm1 * c2) : wi[1];
                    w[2] = near ? R(0) : wi[2];
                    w[3] = near ? wp1 * c2 : wi[3];
                    w[4] = near ? R(0) : wi[4];
                } else if (t < 3 || t > n3 - 2) {
                    const R c2 = ktab<R>(P, 0, t);
                    w[0] = R(0); w[1] = -(wm1 * c2); w[2] = R(0); w[3] = wp1 * c2; w[4] = R(0);
                } else {
                    const bool qk = (ktab<R>(P, 3, t) * fabs(q0[3])) > C.pez_val * mu0;
                    inv_weights(wm2, wm1, w0, wp1, wp2, qk, ktab<R>(P, 1, t), ktab<R>(P, 2, t), w);
                }
                const R czt = ktab<R>(P, 0, t);
                // plane t+2's own-column Q again (in L1 since phase A)
                if (late_qp2 && t + 2 <= n3) {
                    const long long off = (long long)(t + 2) * plane + colo;
#pragma unroll
                    for (int c = 0; c < 5; c++) qp2[c] = (R)ldq_c<PERSIST>(qin() + c * vol + off);
                }
                Fs[0] = Fs[0] + wsum(w, qm2[0], qm1[0], q0[0], sq(iP, 0)[bc], qp2[0]);
                const bool top = t + 1 == n3;   // hD of the top wall plane was staged in the prologue
                // float rings: the top plane's hD from the prologue's staging, under one
                // uniform branch (hp1 is not formed on the top plane, and the march ends
                // there).  Measured with the select weights: 1% faster in the float
                // kernels, 1% slower in the FP64 one (register allocation), which keeps
                // the select inside the flux loop.
#ifdef CHAN_TOP_HOIST_D
                constexpr bool hoist_d = true;
#else
                constexpr bool hoist_d = false;
#endif
#ifdef CHAN_NO_TOP_HOIST_F
                constexpr bool hoist_f = false;
#else
                constexpr bool hoist_f = true;
#endif
                constexpr bool hoist = sizeof(R) == 8 ? hoist_d : hoist_f;
                if (hoist && top) {
#pragma unroll
                    for (int c = 0; c < 4; c++) hp1[c] = (R)P.hwt[c * plane + colo];
                }
#pragma unroll
                for (int c = 1; c < 5; c++) {
                    const R H1 = wsum(w, qm2[c], qm1[c], q0[c], sq(iP, c)[bc], qp2[c]);
                    const R hp = hoist ? hp1[c - 1] : (top ? (R)P.hwt[(c - 1) * plane + colo] : hp1[c - 1]);
                    const R H2 = (hp - hm1[c - 1]) * czt;
                    Fs[c] = (Fs[c] + H1) + H2;
                }
            }
            // source: lagged wall-shear forcing (main_v1.9.f90:565-571), in double
            double src2 = 0.0, src5 = 0.0;
            // FP64 rings: the forcing terms formed on every launch (the statistics
            // array always holds these entries) and selected by the flag, so that the
            // update's block has no branch on it (1.1% of the FP64 stage time);
            // CHAN_FORCE_BRANCH keeps the branch, for measurement
#if defined(CHAN_FORCE_BRANCH)
            constexpr bool force_sel = false;
#elif defined(CHAN_FORCE_SEL_F)
            constexpr bool force_sel = true;
#else
            constexpr bool force_sel = sizeof(R) == 8;
#endif
            if (force_sel) {
                const double tau = P.stat[23 * n3 + 0] - P.stat[23 * n3 + 1];
                const double rb = P.stat[t - 1];
                const double s2 = (0.5 * tau) * rb;
                const double s5 = (((P.ggM * (double)(neb ? um1 : s0.U[bc])) * 0.5) * tau) * rb;
                src2 = P.force_on ? s2 : 0.0;
                src5 = P.force_on ? s5 : 0.0;
            } else if (P.force_on) {
                const double tau = P.stat[23 * n3 + 0] - P.stat[23 * n3 + 1];
                const double rb = P.stat[t - 1];
                src2 = (0.5 * tau) * rb;
                src5 = (((P.ggM * (double)(neb ? um1 : s0.U[bc])) * 0.5) * tau) * rb;
            }
            double Rd[5];
            Rd[0] = -(double)Fs[0];
            Rd[1] = src2 - (double)Fs[1];
            Rd[2] = -(double)Fs[2];
            Rd[3] = -(double)Fs[3];
            if (buoy) {
                // buoyancy on the wall-normal momentum and its work on the energy
                const double bq = P.ri * ((double)q0[0] * ((double)(neb ? T0n : s0.T[bc]) - P.tref));
                Rd[3] = bq - (double)Fs[3];
                src5 = src5 + (P.ggM * (double)(neb ? w0n : s0.W[bc])) * bq;
            }
            Rd[4] = src5 - (double)Fs[4];
            // RK update in double, on the stage input at its stored precision
            double qs[5];
            if (std::is_same<QI, R>::value) {
#pragma unroll
                for (int c = 0; c < 5; c++) qs[c] = (double)q0[c];
            } else {
                const long long off = (long long)t * plane + colo;
#pragma unroll
                for (int c = 0; c < 5; c++) qs[c] = ldq_c<PERSIST>(qin() + c * vol + off);
            }
            double qn[5];
            double qb[5] = {0, 0, 0, 0, 0};
            if (P.rk_mode != 0) {
                if (S::tma_base) {
#pragma unroll
                    for (int c = 0; c < 5; c++) qb[c] = sQB[c * NT + tid];
                } else if (S::prefetch_base) {
                    cp_async_wait<0>();
#pragma unroll
                    for (int c = 0; c < 5; c++) qb[c] = sQB[c * NT + tid];
                } else {
#ifdef CHAN_EARLY_BASE
#pragma unroll
                    for (int c = 0; c < 5; c++) qb[c] = qbe[c];
#else
                    const long long off = (long long)t * plane + colo;
#pragma unroll
                    for (int c = 0; c < 5; c++) qb[c] = ldq_c<PERSIST>(P.qbase + c * vol + off);
#endif
                }
            }
            if (P.rk_mode == 0) {
#pragma unroll
                for (int c = 0; c < 5; c++) qn[c] = qs[c] + P.rk_cdt * Rd[c];
            } else if (P.rk_mode == 1) {
#pragma unroll
                for (int c = 0; c < 5; c++) qn[c] = qb[c] + P.rk_cdt * Rd[c];
            } else {
#pragma unroll
                for (int c = 0; c < 5; c++) qn[c] = (P.rk_a * qb[c] + P.rk_b * qs[c]) + P.rk_cdt * Rd[c];
            }
            // store + periodic images (the ghosts the reference's halo exchange fills)
            const int im = (i <= 3) ? i + (n1 - 2) : ((i >= n1 - 2) ? i - (n1 - 2) : -1);
            const int jm = (j <= 3) ? j + (n2 - 2) : ((j >= n2 - 2) ? j - (n2 - 2) : -1);
            const long long pk = (long long)t * plane;
            // FP64 rings: the periodic images under one branch that only points within 2
            // of a periodic edge take (0.7% of the stage time); the float rings keep
            // predicated stores (the branch costs them spills)
#ifndef CHAN_NO_IMAGE_BRANCH
            constexpr bool img_branch = sizeof(R) == 8;
#else
            constexpr bool img_branch = false;
#endif
            if (img_branch) {
                // own point; then, only at points within 2 of a periodic edge, the images
#pragma unroll
                for (int c = 0; c < 5; c++) qout()[c * vol + pk + colo] = (QO)qn[c];
                if (im >= 0 || jm >= 0) {
#pragma unroll
                    for (int c = 0; c < 5; c++) {
                        QO *O = qout() + c * vol + pk;
                        const QO v = (QO)qn[c];
                        if (im >= 0) O[(long long)j * P.px + im] = v;
                        if (jm >= 0) O[(long long)jm * P.px + i] = v;
                        if (im >= 0 && jm >= 0) O[(long long)jm * P.px + im] = v;
                    }
                }
            } else {
#pragma unroll
                for (int c = 0; c < 5; c++) {
                    QO *O = qout() + c * vol + pk;
                    const QO v = (QO)qn[c];
                    O[(long long)j * P.px + i] = v;
                    if (im >= 0) O[(long long)j * P.px + im] = v;
                    if (jm >= 0) O[(long long)jm * P.px + i] = v;
                    if (im >= 0 && jm >= 0) O[(long long)jm * P.px + im] = v;
                }
            }
            if (P.check) {
                const double tr = qn[0] * qn[4] - P.ggMh * ((qn[1] * qn[1] + qn[2] * qn[2]) + qn[3] * qn[3]);
                if (qn[0] < 0.0 || (qn[0] > 0.0 && tr < 0.0)) flag_blown(P.status, i, j, t, kstep(P));
                bool fin = true;
#pragma unroll
                for (int c = 0; c < 5; c++) fin = fin && isfinite(qn[c]);
                if (!fin) flag_nonfinite(P.status, i, j, t);
            }
        }
        // ---------- F: plane t becomes t-1; rotate the rings (no barrier: see neb)
#pragma unroll
        for (int c = 0; c < 5; c++) {
            qm2[c] = qm1[c];
            qm1[c] = q0[c];
        }
        wm2 = wm1;
        if (neb) {
            wm1 = w0n;
        } else {
            um1 = s0.U[bc]; vm1 = s0.V[bc]; wm1 = s0.W[bc];
            keep_halo(s0);
        }
#pragma unroll
        for (int c = 0; c < 4; c++) {
            hm1[c] = h0[c];
            h0[c] = hp1[c];
        }
        {
            const int o = iZ;
            iZ = iP; iP = iN; iN = o;
            int x = pZ; pZ = pP; pP = x;
            x = mZ; mZ = mP; mP = x;
        }
        if (!neb) __syncthreads();
    }
    if (S::prefetch_base) cp_async_wait<0>();
}

template <int TI, int TJ, typename QI, typename QO, typename R, bool BUOY>
__global__ void __launch_bounds__(TI *TJ, StageShape<TI, TJ, R>::minb)
    k_stage(const KParams P, const __grid_constant__ CUtensorMap tmq, const __grid_constant__ CUtensorMap tmb)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    stage_body<TI, TJ, QI, QO, R, BUOY ? 1 : 0, false>(P, &tmq, &tmb, blockIdx.x, blockIdx.y, blockIdx.z,
                                                          threadIdx.x, threadIdx.y, smem_raw);
}

// ---------------------------------------------------------------------------
// Wall BC + pressure BC (main_v1.9.f90:623-720 on the two wall planes).
// One thread per (i,j) of a wall plane, ghosts included.

// var(u, v, T) of an interior point as the reference holds it (corner columns
// keep their stale values)
template <typename QT>
__device__ __forceinline__ void inner_uvT(const KParams &P, int i, int j, int k, double &u, double &v, double &T)
{
    const QT *qo = static_cast<const QT *>(P.qout);
    const int n1 = P.n1, n2 = P.n2;
    if ((i == 1 || i == n1) && (j == 1 || j == n2)) {
        const double *C = P.cs + ((size_t)k * 4 + (i == 1 ? 0 : 1) + (j == 1 ? 0 : 2)) * 7;
        u = C[1]; v = C[2]; T = C[5];
        return;
    }
    const long long o = (long long)k * P.plane + (long long)j * P.px + i;
    const double q0 = qo[o];
#ifndef CHAN_TRUE_DIV
    const double r = rcp_fast(q0);
    u = (double)qo[P.vol + o] * r;
    v = (double)qo[2 * P.vol + o] * r;
    const double w = (double)qo[3 * P.vol + o] * r;
    const double E = (double)qo[4 * P.vol + o] * r;
#else
    u = (double)qo[P.vol + o] / q0;
    v = (double)qo[2 * P.vol + o] / q0;
    const double w = (double)qo[3 * P.vol + o] / q0;
    const double E = (double)qo[4 * P.vol + o] / q0;
#endif
    T = E - P.ggMh * ((u * u + v * v) + w * w);
}

// wall values u, v, T of point (i,j) of wall `wall` after the wall BC
template <typename QT>
__device__ void wall_point(const KParams &P, int wall, int i, int j, double &u, double &v, double &T)
{
    const WallBC &B = P.wbc[wall];
    const int n1 = P.n1, n2 = P.n2;
    const int ic = i < 1 ? 1 : (i > n1 ? n1 : i), jc = j < 1 ? 1 : (j > n2 ? n2 : j);
    const int k2 = wall == 0 ? 2 : P.n3 - 1, k3 = wall == 0 ? 3 : P.n3 - 2;
    const double *c = wall == 0 ? P.f1 : P.b1;
    u = 0.0;
    v = 0.0;
    double u2 = 0, v2 = 0, T2 = 0, u3 = 0, v3 = 0, T3 = 0;
    const bool need_inner = (B.vel == 1 && B.mask[(jc - 1) * n1 + ic - 1]) || B.therm == 1;
    if (need_inner) {
        inner_uvT<QT>(P, ic, jc, k2, u2, v2, T2);
        inner_uvT<QT>(P, ic, jc, k3, u3, v3, T3);
    }
    if (B.vel == 1) {
        if (B.mask[(jc - 1) * n1 + ic - 1]) {
            u = ((B.g - c[1] * u2) - c[2] * u3) / c[0];
            v = ((B.g - c[1] * v2) - c[2] * v3) / c[0];
        }
    } else if (B.vel == 2) {
        u = B.uv[(jc - 1) * n1 + ic - 1];
        v = B.uv[n1 * n2 + (jc - 1) * n1 + ic - 1];
    } else if (B.vel == 3) {
        const double x = B.x1[ic - 1];
        v = B.A * sin((B.kx * x + B.om * ktime(P)) + ((jc & 1) ? B.ph : 0.0));
    }
    T = (B.therm == 1) ? ((B.dTdz - c[1] * T2) - c[2] * T3) / c[0] : B.Tw;
}

// QT: storage type of the stage output the wall BC reads (the planes next to the wall)
constexpr int kWallBX = 32, kWallBY = 8;
constexpr int kWallHX = kWallBX + 2, kWallHY = kWallBY + 2;
using WallStage = double[2][6][kWallHY][kWallHX];

// One block's work of the wall kernel: block (bx, by) of wall `wall`,
// thread (tx, ty), near-wall staging area sp.
template <typename QT>
__device__ __forceinline__ void wall_body(const KParams &P, int bx_, int by_, int wall, int tx, int ty, WallStage &sp)
{
    const QT *qo = static_cast<const QT *>(P.qout);
    const int i = bx_ * kWallBX + tx;
    const int j = by_ * kWallBY + ty;
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3;
    const long long plane = P.plane, vol = P.vol;
    // primitives of the two planes next to the wall on the block's (i,j) tile
    // plus a 1-point halo, each computed once: [plane][r,u,v,w,p,mu][by][bx]
    constexpr int HX = kWallHX, HY = kWallHY;
    {
        const int k2 = wall == 0 ? 2 : n3 - 1, k3 = wall == 0 ? 3 : n3 - 2;
        const int i0 = bx_ * kWallBX - 1, j0 = by_ * kWallBY - 1;
        for (int e = ty * kWallBX + tx; e < 2 * HX * HY; e += kWallBX * kWallBY) {
            const int pl = e / (HX * HY), r0 = e - pl * HX * HY, by = r0 / HX, bx = r0 - by * HX;
            const int ii = i0 + bx, jj = j0 + by;
            if (ii < 1 || ii > n1 || jj < 1 || jj > n2) continue;
            const long long o = (long long)(pl == 0 ? k2 : k3) * plane + (long long)jj * P.px + ii;
            const double q0 = qo[o], q1 = qo[vol + o], q2 = qo[2 * vol + o];
            const double q3 = qo[3 * vol + o], q4 = qo[4 * vol + o];
#ifndef CHAN_TRUE_DIV
            const double r = rcp_fast(q0);
            const double u = q1 * r, v = q2 * r, w = q3 * r;
            const double E = q4 * r;
#else
            const double u = q1 / q0, v = q2 / q0, w = q3 / q0;
            const double E = q4 / q0;
#endif
            const double T = E - P.ggMh * ((u * u + v * v) + w * w);
            sp[pl][0][by][bx] = q0;
            sp[pl][1][by][bx] = u;
            sp[pl][2][by][bx] = v;
            sp[pl][3][by][bx] = w;
#ifndef CHAN_TRUE_DIV
            sp[pl][4][by][bx] = (q0 * T) * P.inv_gM2;
#else
            sp[pl][4][by][bx] = (q0 * T) / P.gM2;
#endif
            sp[pl][5][by][bx] = pow07(T);
        }
    }
    __syncthreads();
    if (i > n1 + 1 || j > n2 + 1) return;
    if (frozen(P.status, kstep(P))) return;
    double *W = P.wp + (size_t)wall * 8 * plane;
    const long long idx = (long long)j * P.px + i;
    const bool custom = P.wall_custom != 0;
    double uw = 0.0, vw = 0.0, Tw = wall == 0 ? P.Twb : P.Twt;
    double muw = wall == 0 ? P.muwb : P.muwt;
    if (custom) {
        wall_point<QT>(P, wall, i, j, uw, vw, Tw);
        if (P.wbc[wall].therm == 1) muw = pow07(Tw);
    }
    const double pold = W[6 * plane + idx];
    const double rho = (P.gM2 * pold) / Tw;   // gama*Mac**2*p/T with the previous p
    double pnew = pold;
    if (i >= 2 && i <= n1 - 1 && j >= 2 && j <= n2 - 1) {
        // neighbours at the two planes next to the wall: k2 (adjacent) and k3
        const int k2 = wall == 0 ? 2 : n3 - 1, k3 = wall == 0 ? 3 : n3 - 2;
        const double *c1 = wall == 0 ? P.f1 : P.b1;
        const double *c2 = wall == 0 ? P.f2 : P.b2;
        // primitive + mu of one interior point, as calcPrim/calcBC produce them
        // (staged above); kk selects the plane k2 or k3
        auto prim = [&](int ii, int jj, int kk, double &r, double &u, double &v, double &w, double &T,
                        double &p, double &mu) {
            const int pl = kk == k2 ? 0 : 1;
            const int bx = ii - bx_ * kWallBX + 1, by = jj - by_ * kWallBY + 1;
            r = sp[pl][0][by][bx];
            u = sp[pl][1][by][bx];
            v = sp[pl][2][by][bx];
            w = sp[pl][3][by][bx];
            p = sp[pl][4][by][bx];
            mu = sp[pl][5][by][bx];
            T = 0.0;
        };
        // wall-point terms c0*mu_w*u_w of the neighbours (zero for a no-slip wall)
        double t_ip = 0.0, t_im = 0.0, t_jp = 0.0, t_jm = 0.0;
        if (custom) {
            double u, v, T;
            wall_point<QT>(P, wall, i + 1, j, u, v, T);
            t_ip = c1[0] * (P.wbc[wall].therm == 1 ? pow07(T) : muw) * u;
            wall_point<QT>(P, wall, i - 1, j, u, v, T);
            t_im = c1[0] * (P.wbc[wall].therm == 1 ? pow07(T) : muw) * u;
            wall_point<QT>(P, wall, i, j + 1, u, v, T);
            t_jp = c1[0] * (P.wbc[wall].therm == 1 ? pow07(T) : muw) * v;
            wall_point<QT>(P, wall, i, j - 1, u, v, T);
            t_jm = c1[0] * (P.wbc[wall].therm == 1 ? pow07(T) : muw) * v;
        }
        double r, u, v, w, T, p, mu;
        double a2, a3, b2, b3;
        // d/dx of mu*du/dz
        prim(i + 1, j, k2, r, u, v, w, T, p, mu); a2 = c1[1] * mu * u;
        prim(i + 1, j, k3, r, u, v, w, T, p, mu); a3 = c1[2] * mu * u;
        prim(i - 1, j, k2, r, u, v, w, T, p, mu); b2 = c1[1] * mu * u;
        prim(i - 1, j, k3, r, u, v, w, T, p, mu); b3 = c1[2] * mu * u;
        const double dudxdz = (((t_ip + a2) + a3) - ((t_im + b2) + b3)) * P.hdx;
        prim(i, j + 1, k2, r, u, v, w, T, p, mu); a2 = c1[1] * mu * v;
        prim(i, j + 1, k3, r, u, v, w, T, p, mu); a3 = c1[2] * mu * v;
        prim(i, j - 1, k2, r, u, v, w, T, p, mu); b2 = c1[1] * mu * v;
        prim(i, j - 1, k3, r, u, v, w, T, p, mu); b3 = c1[2] * mu * v;
        const double dvdydz = (((t_jp + a2) + a3) - ((t_jm + b2) + b3)) * P.hdy;
        double p2, p3, d2, d3, e2, e3;
        prim(i, j, k2, r, u, v, w, T, p, mu);
        d2 = c2[1] * mu * w; e2 = c1[1] * r * (w * w); p2 = p;
        prim(i, j, k3, r, u, v, w, T, p, mu);
        d3 = c2[2] * mu * w; e3 = c1[2] * r * (w * w); p3 = p;
        // the wall-point w terms vanish: w = 0 on every wall
        const double d2wdz2 = d2 + d3;
        const double drhow2dz = e2 + e3;
        const double lhs = P.invRe * ((-dudxdz - dvdydz) + P.two3rd * ((dudxdz + dvdydz) - 2.0 * d2wdz2)) + drhow2dz;
        pnew = -((lhs + c1[1] * p2) + c1[2] * p3) / c1[0];
    }
    W[0 * plane + idx] = rho;
    W[1 * plane + idx] = uw;
    W[2 * plane + idx] = vw;
    W[3 * plane + idx] = 0.0;
    W[4 * plane + idx] = custom ? Tw + P.ggMh * ((uw * uw + vw * vw) + 0.0) : Tw;
    W[5 * plane + idx] = Tw;
    W[6 * plane + idx] = pnew;
    W[7 * plane + idx] = muw;
    if (P.check && i >= 1 && i <= n1 && j >= 1 && j <= n2) {
        if (rho < 0.0 || Tw < 0.0) flag_blown(P.status, i, j, wall == 0 ? 1 : n3, kstep(P));
        if (!isfinite(rho) || !isfinite(pnew)) flag_nonfinite(P.status, i, j, wall == 0 ? 1 : n3);
    }
}

template <typename QT>
__global__ void __launch_bounds__(kWallBX * kWallBY) k_wall(const KParams P)
{
    __shared__ double sp[2][6][kWallHY][kWallHX];
    wall_body<QT>(P, blockIdx.x, blockIdx.y, blockIdx.z, threadIdx.x, threadIdx.y, sp);
}

// ---------------------------------------------------------------------------
// var(i,j,k,1:7) as the reference holds it after a stage (used by the
// statistics, the blow-up scan and downloads).
__device__ __forceinline__ void ref_var(const KParams &P, const double *q, int i, int j, int k, double x[7])
{
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3;
    if (k == 1 || k == n3) {
        const double *W = P.wp + (size_t)(k == 1 ? 0 : 8) * P.plane + (long long)j * P.px + i;
        x[0] = W[0]; x[1] = W[P.plane]; x[2] = W[2 * P.plane]; x[3] = W[3 * P.plane];
        x[4] = W[4 * P.plane]; x[5] = W[5 * P.plane]; x[6] = W[6 * P.plane];
        return;
    }
    const bool ci = (i == 1 || i == n1), cj = (j == 1 || j == n2);
    if (ci && cj) {
        const int c = (i == 1 ? 0 : 1) + (j == 1 ? 0 : 2);
        const double *C = P.cs + ((size_t)k * 4 + c) * 7;
#pragma unroll
        for (int m = 0; m < 7; m++) x[m] = C[m];
        return;
    }
    const long long o = (long long)k * P.plane + (long long)j * P.px + i;
    const double q0 = q[o];
    x[0] = q0;
#ifndef CHAN_TRUE_DIV
    // one reciprocal for the four quotients (within an ulp or two of them; the
    // four true divisions, CHAN_TRUE_DIV, cost 0.65% of the step in this and the
    // wall kernel)
    const double r = rcp_fast(q0);
    x[1] = q[P.vol + o] * r;
    x[2] = q[2 * P.vol + o] * r;
    x[3] = q[3 * P.vol + o] * r;
    x[4] = q[4 * P.vol + o] * r;
    x[5] = x[4] - P.ggMh * ((x[1] * x[1] + x[2] * x[2]) + x[3] * x[3]);
    x[6] = (x[0] * x[5]) * P.inv_gM2;
#else
    x[1] = q[P.vol + o] / q0;
    x[2] = q[2 * P.vol + o] / q0;
    x[3] = q[3 * P.vol + o] / q0;
    x[4] = q[4 * P.vol + o] / q0;
    x[5] = x[4] - P.ggMh * ((x[1] * x[1] + x[2] * x[2]) + x[3] * x[3]);
    x[6] = (x[0] * x[5]) / P.gM2;
#endif
}

// Plane moments (avgSpatial, main_v1.9.f90:995-1025) and wall shear
// (calcTauWall, main_v1.9.f90:930-977), in two passes.
constexpr int kStatThreads = 256;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Pass 1: block (pb, sub) sums the points sub, sub+S, ... (in units of
// kStatThreads) of plane pb (pb < n3: the 23 moment sums of plane k = pb+1;
// pb = n3, n3+1: the wall-shear sum of the bottom, top wall) into
// part[(pb*S + sub)*23 + c].  Pass 2 adds the S partial sums in a fixed
// order: the result is deterministic.
using StatRed = double[kStatThreads / 32][23];
__device__ __forceinline__ void stats_part_body(const KParams &P, const double *q, int do_moments, int do_tau, int S,
                                                double *part, int blk, int tid, StatRed &red)
{
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3;
    const int pb = blk / S, sub = blk - pb * S;
    const int lane = tid & 31, warp = tid >> 5;
    if (frozen(P.status, kstep(P) + 1)) return;
    double *out = part + ((size_t)pb * S + sub) * 23;
    if (pb < n3) {
        if (!do_moments) return;
        const int k = pb + 1;
        double acc[23];
#pragma unroll
        for (int c = 0; c < 23; c++) acc[c] = 0.0;
        const int np = n1 * n2;
#pragma unroll 2
        for (int p = sub * kStatThreads + tid; p < np; p += S * kStatThreads) {
            const int jj = p / n1, ii = p - jj * n1;
            double x[7];
            ref_var(P, q, ii + 1, jj + 1, k, x);
#pragma unroll
            for (int m = 0; m < 7; m++) {
                acc[m] += x[m];
                acc[7 + m] += x[m] * x[m];
            }
            acc[14] += x[0] * x[3];
            acc[15] += x[0] * x[5];
            acc[16] += x[1] * x[2];
            acc[17] += x[1] * x[3];
            acc[18] += x[2] * x[3];
            acc[19] += x[2] * x[5];
            acc[20] += x[5] * x[3];
            acc[21] += x[6] * x[3];
            acc[22] += x[6] * x[5];
        }
#pragma unroll
        for (int c = 0; c < 23; c++) {
            const double s = warp_sum(acc[c]);
            if (lane == 0) red[warp][c] = s;
        }
        __syncthreads();
        if (tid < 23) {
            double s = 0.0;
            for (int w = 0; w < kStatThreads / 32; w++) s += red[w][tid];
            out[tid] = s;
        }
        return;
    }
    if (!do_tau) return;
    const int wall = pb - n3;
    const double *W = P.wp + (size_t)wall * 8 * P.plane;
    const double *c = wall == 0 ? P.f1 : P.b1;
    const int k2 = wall == 0 ? 2 : n3 - 1, k3 = wall == 0 ? 3 : n3 - 2;
    double acc = 0.0;
    const int ni = n1 - 2, np = (n1 - 2) * (n2 - 2);
    for (int p = sub * kStatThreads + tid; p < np; p += S * kStatThreads) {
        const int jj = 2 + p / ni, ii = 2 + p % ni;
        const long long o = (long long)jj * P.px + ii;
        const double mu = W[7 * P.plane + o];
        const double dwdx = ((mu * (W[3 * P.plane + o + 1] - W[3 * P.plane + o - 1])) * 0.5) * P.invdx;
        const long long o2 = (long long)k2 * P.plane + o, o3 = (long long)k3 * P.plane + o;
        const double u2 = q[P.vol + o2] / q[o2];
        const double u3 = q[P.vol + o3] / q[o3];
        const double dudz = mu * ((c[0] * W[1 * P.plane + o] + c[1] * u2) + c[2] * u3);
        acc += (dwdx + dudz) * P.invRe;
    }
    const double s = warp_sum(acc);
    if (lane == 0) red[warp][0] = s;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < kStatThreads / 32; w++) t += red[w][0];
        out[0] = t;
    }
}

__global__ void __launch_bounds__(kStatThreads, 3) k_stats_part(const KParams P, const double *q, int do_moments,
                                                             int do_tau, int S, double *part)
{
    __shared__ double red[kStatThreads / 32][23];
    stats_part_body(P, q, do_moments, do_tau, S, part, blockIdx.x, threadIdx.x, red);
}

// Pass 2: one warp per plane / wall adds the S partial sums in order and
// writes stat1Spc, stat2Spc, corrSpc (divided by nP1*nP2) and tauL, tauU
// (divided by (nP1-2)*(nP2-2)); with time averaging on, also adds them into tacc.
__device__ __forceinline__ void stats_fin_body(const KParams &P, int do_moments, int do_tau, int S, const double *part,
                                               int pb, int c)
{
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3;
    if (frozen(P.status, kstep(P) + 1)) return;
    const double *in = part + (size_t)pb * S * 23;
    if (pb < n3) {
        if (!do_moments || c >= 23) return;
        double s = 0.0;
        for (int u = 0; u < S; u++) s += in[(size_t)u * 23 + c];
        const double nxy = (double)(n1 * n2);
        double *out;
        if (c < 7) out = P.stat + (size_t)c * n3;
        else if (c < 14) out = P.stat + (size_t)7 * n3 + (size_t)(c - 7) * n3;
        else out = P.stat + (size_t)14 * n3 + (size_t)(c - 14) * n3;
        const double val = s / nxy;
        out[pb] = val;
        if (P.acc_on) P.tacc[(out - P.stat) + pb] += val;
        return;
    }
    if (!do_tau || c != 0) return;
    const int wall = pb - n3;
    double s = 0.0;
    for (int u = 0; u < S; u++) s += in[(size_t)u * 23];
    const double val = s / (double)((n1 - 2) * (n2 - 2));
    P.stat[(size_t)23 * n3 + wall] = val;
    if (P.acc_on) P.tacc[(size_t)23 * n3 + wall] += val;
}

__global__ void k_stats_fin(const KParams P, int do_moments, int do_tau, int S, const double *part)
{
    stats_fin_body(P, do_moments, do_tau, S, part, blockIdx.x, threadIdx.x);
}

// ---------------------------------------------------------------------------
// Diagnostics series (main_v1.9.f90:799-906), every `every` steps:
//   KE = sum over all stored points of (u^2+v^2)+w^2, divided by nP1*nP2*nP3;
//   bulk rho, u and rho*u through the x-planes i = plane(n): over the cells
//   j=1..nP2-1, k=1..nP3-1 the mean of the four corner values times
//   dAyz = dy*(x3(k+1)-x3(k)), summed and divided by Ayz = x3(nP3)*x2(nP2).
// A plane outside 3..nP1-2 gives 0 (the single-rank form of the reference's
// plane(i) > bn(1) .and. plane(i) < en(1) test).  Record layout:
//   [nstep, time, KE, rho_b[np], U_b[np], rhoU_b[np]]
// nstep is -1 when a blow-up stopped the run before that step's diagnostics.
constexpr int kDiagMaxPlanes = 8;

struct DiagParams {
    int nplanes;
    int planes[kDiagMaxPlanes];
    const double *x3q;   // x3 as the diagnostics see it (the deck's F10.6 column after a restart)
    double dy, Ayz;
    double *part;        // nP3 per-plane KE sums
};

__global__ void __launch_bounds__(kStatThreads) k_diag_ke(const KParams P, const double *q, const DiagParams D)
{
    __shared__ double red[kStatThreads / 32];
    const int n1 = P.n1, n2 = P.n2;
    const int k = blockIdx.x + 1, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (frozen(P.status, kstep(P) + 1)) return;
    double acc = 0.0;
    const int np = n1 * n2;
    for (int p = tid; p < np; p += kStatThreads) {
        const int jj = p / n1, ii = p - jj * n1;
        double x[7];
        ref_var(P, q, ii + 1, jj + 1, k, x);
        acc += (x[1] * x[1] + x[2] * x[2]) + x[3] * x[3];
    }
    const double s = warp_sum(acc);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < kStatThreads / 32; w++) t += red[w];
        D.part[k - 1] = t;
    }
}

// block 0: KE from the per-plane sums; block 1+n*np+m: quantity n at plane m
__global__ void __launch_bounds__(kStatThreads) k_diag_fin(const KParams P, const double *q, const DiagParams D,
                                                           double *rec, double time)
{
    __shared__ double red[kStatThreads / 32];
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3;
    const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (frozen(P.status, kstep(P) + 1)) {
        if (b == 0 && tid == 0) rec[0] = -1.0;
        return;
    }
    if (b == 0) {
        if (tid == 0) {
            double t = 0.0;
            for (int k = 0; k < n3; k++) t += D.part[k];
            rec[0] = (double)kstep(P);
            rec[1] = time;
            rec[2] = t / ((double)n1 * (double)n2 * (double)n3);
        }
        return;
    }
    const int qn = (b - 1) / D.nplanes, m = (b - 1) % D.nplanes;
    const int ip = D.planes[m];
    double acc = 0.0;
    if (ip > 2 && ip < n1 - 1) {
        const int nj = n2 - 1, ncell = (n2 - 1) * (n3 - 1);
        for (int c = tid; c < ncell; c += kStatThreads) {
            const int j = 1 + c % nj, k = 1 + c / nj;
            double a[7], bb[7], cc[7], d[7];
            ref_var(P, q, ip, j, k, a);
            ref_var(P, q, ip, j + 1, k, bb);
            ref_var(P, q, ip, j, k + 1, cc);
            ref_var(P, q, ip, j + 1, k + 1, d);
            double f0, f1, f2, f3;
            if (qn == 0) { f0 = a[0]; f1 = bb[0]; f2 = cc[0]; f3 = d[0]; }
            else if (qn == 1) { f0 = a[1]; f1 = bb[1]; f2 = cc[1]; f3 = d[1]; }
            else { f0 = a[0] * a[1]; f1 = bb[0] * bb[1]; f2 = cc[0] * cc[1]; f3 = d[0] * d[1]; }
            const double dAyz = D.dy * (D.x3q[k] - D.x3q[k - 1]);
            acc += (0.25 * (((f0 + f1) + f2) + f3)) * dAyz;
        }
    }
    const double s = warp_sum(acc);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < kStatThreads / 32; w++) t += red[w];
        rec[3 + qn * D.nplanes + m] = t / D.Ayz;
    }
}

// fluctuation field var(i,j,k,:) - mean(k,:) (fluc.f90:63-69), in place on a
// [7][N] device copy of var
__global__ void k_fluctuation(double *var, const double *mean, int n1, int n2, int n3)
{
    const long long N = (long long)n1 * n2 * n3;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
         p += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(p / ((long long)n1 * n2));
#pragma unroll
        for (int m = 0; m < 7; m++) var[(size_t)m * N + p] -= mean[(size_t)m * n3 + k];
    }
}

// Q-criterion of a velocity field (qInvariant.f90:26-81): central differences
// on the non-uniform coordinates x, y, z; Q = (P^2 - sum S^2 + sum R^2)/2 with
// P = -trace(J), S and R the symmetric and antisymmetric parts of J.  Points
// on the box faces get 0.  u, v, w and Q are [k][j][i].
__global__ void k_qcrit(int n1, int n2, int n3, const double *u, const double *v, const double *w,
                        const double *x, const double *y, const double *z, double *Q)
{
    const long long N = (long long)n1 * n2 * n3;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
         p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % n1);
        const int j = (int)((p / n1) % n2);
        const int k = (int)(p / ((long long)n1 * n2));
        if (i == 0 || i == n1 - 1 || j == 0 || j == n2 - 1 || k == 0 || k == n3 - 1) {
            Q[p] = 0.0;
            continue;
        }
        const long long si = 1, sj = n1, sk = (long long)n1 * n2;
        const double dx1 = x[i + 1] - x[i], dx2 = x[i] - x[i - 1];
        const double dy1 = y[j + 1] - y[j], dy2 = y[j] - y[j - 1];
        const double dz1 = z[k + 1] - z[k], dz2 = z[k] - z[k - 1];
        const double *U[3] = {u, v, w};
        double J[3][3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const double *f = U[c];
            const double f0 = f[p];
            J[c][0] = ((dx2 / dx1) * (f[p + si] - f0) + (dx1 / dx2) * (f0 - f[p - si])) / (dx1 + dx2);
            J[c][1] = ((dy2 / dy1) * (f[p + sj] - f0) + (dy1 / dy2) * (f0 - f[p - sj])) / (dy1 + dy2);
            J[c][2] = ((dz2 / dz1) * (f[p + sk] - f0) + (dz1 / dz2) * (f0 - f[p - sk])) / (dz1 + dz2);
        }
        // sum(S**2) and sum(-R**2) in column-major order
        double as1 = 0.0, as2 = 0.0;
#pragma unroll
        for (int cj = 0; cj < 3; cj++)
#pragma unroll
            for (int ci = 0; ci < 3; ci++) {
                const double sv = ci == cj ? J[ci][ci] : 0.5 * (J[ci][cj] + J[cj][ci]);
                const double rv = ci == cj ? 0.0 : 0.5 * (J[ci][cj] - J[cj][ci]);
                as1 += sv * sv;
                as2 += -(rv * rv);
            }
        const double P_ = -((J[0][0] + J[1][1]) + J[2][2]);
        Q[p] = 0.5 * ((P_ * P_ - as1) - as2);
    }
}

// ---------------------------------------------------------------------------
// Upload: var(1:nP1,1:nP2,1:nP3,1:7) (device copy, [m][k][j][i]) -> state.
// initSolV (main_v1.9.f90:284-294): Q = rho*(1,u,v,w,E) at every point.
__global__ void k_upload(const KParams P, const double *var, double *qa, double *qb, double *qc, double *cs)
{
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3;
    const long long N = (long long)n1 * n2 * n3;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
         p += (long long)gridDim.x * blockDim.x) {
        const int ii = (int)(p % n1);
        const int jj = (int)((p / n1) % n2);
        const int kk = (int)(p / ((long long)n1 * n2));
        const int i = ii + 1, j = jj + 1, k = kk + 1;
        // T and p (columns 5, 6) are read only on the wall planes and the
        // corner columns: the upload copies them only there
        const bool wall = (k == 1 || k == n3), corner = (i == 1 || i == n1) && (j == 1 || j == n2);
        double x[7];
#pragma unroll
        for (int m = 0; m < 5; m++) x[m] = var[(size_t)m * N + p];
        x[5] = (wall || corner) ? var[(size_t)5 * N + p] : 0.0;
        x[6] = (wall || corner) ? var[(size_t)6 * N + p] : 0.0;
        const long long o = (long long)k * P.plane + (long long)j * P.px + i;
        double q[5] = {x[0], x[0] * x[1], x[0] * x[2], x[0] * x[3], x[0] * x[4]};
#pragma unroll
        for (int c = 0; c < 5; c++) qa[c * P.vol + o] = q[c];
        if (k == 1 || k == n3) {
#pragma unroll
            for (int c = 0; c < 5; c++) {
                qb[c * P.vol + o] = q[c];
                if (qc) qc[c * P.vol + o] = q[c];
            }
            double *W = P.wp + (size_t)(k == 1 ? 0 : 8) * P.plane + (long long)j * P.px + i;
#pragma unroll
            for (int m = 0; m < 7; m++) W[(size_t)m * P.plane] = x[m];
            W[(size_t)7 * P.plane] = pow(x[5], 0.7);
        } else if ((i == 1 || i == n1) && (j == 1 || j == n2)) {
            const int c = (i == 1 ? 0 : 1) + (j == 1 ? 0 : 2);
#pragma unroll
            for (int m = 0; m < 7; m++) cs[((size_t)k * 4 + c) * 7 + m] = x[m];
        }
    }
}

// periodic images of Q for interior planes (the reference's initial share2P,
// including corner images so every periodic read is consistent); and of the
// wall planes' primitive ring i,j in {0, nP+1}

__global__ void k_fill_ghosts(const KParams P, double *q)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 2 + blockIdx.z;
    const int n1 = P.n1, n2 = P.n2;
    if (i > n1 + 1 || j > n2 + 1) return;
    const int si = wrap_idx(i, n1), sj = wrap_idx(j, n2);
    if (si == i && sj == j) return;
    const long long o = (long long)k * P.plane + (long long)j * P.px + i;
    const long long s = (long long)k * P.plane + (long long)sj * P.px + si;
#pragma unroll
    for (int c = 0; c < 5; c++) q[c * P.vol + o] = q[c * P.vol + s];
}

__global__ void k_fill_wall_ring(const KParams P)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int wall = blockIdx.z;
    const int n1 = P.n1, n2 = P.n2;
    if (i > n1 + 1 || j > n2 + 1) return;
    if (i >= 1 && i <= n1 && j >= 1 && j <= n2) return;
    const int si = (i == 0 || i == n1 + 1) ? wrap_idx(i, n1) : i;
    const int sj = (j == 0 || j == n2 + 1) ? wrap_idx(j, n2) : j;
    double *W = P.wp + (size_t)wall * 8 * P.plane;
#pragma unroll
    for (int m = 0; m < 8; m++)
        W[(size_t)m * P.plane + (long long)j * P.px + i] = W[(size_t)m * P.plane + (long long)sj * P.px + si];
}

// Download: state -> var(1:nP1,1:nP2,1:nP3,1:7) ([m][k][j][i])
__global__ void k_download(const KParams P, const double *q, double *var)
{
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3;
    const long long N = (long long)n1 * n2 * n3;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
         p += (long long)gridDim.x * blockDim.x) {
        const int ii = (int)(p % n1);
        const int jj = (int)((p / n1) % n2);
        const int kk = (int)(p / ((long long)n1 * n2));
        double x[7];
        ref_var(P, q, ii + 1, jj + 1, kk + 1, x);
#pragma unroll
        for (int m = 0; m < 7; m++) var[(size_t)m * N + p] = x[m];
    }
}

// checkSoln over every point (main_v1.9.f90:729-740)
__global__ void k_check(const KParams P, const double *q)
{
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3;
    const long long N = (long long)n1 * n2 * n3;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
         p += (long long)gridDim.x * blockDim.x) {
        const int ii = (int)(p % n1);
        const int jj = (int)((p / n1) % n2);
        const int kk = (int)(p / ((long long)n1 * n2));
        double x[7];
        ref_var(P, q, ii + 1, jj + 1, kk + 1, x);
        if (x[0] < 0.0 || x[5] < 0.0) flag_blown(P.status, ii + 1, jj + 1, kk + 1, kstep(P));
    }
}

// ---------------------------------------------------------------------------
// Learned subgrid closure: features, filtered-DNS targets, and the closure
// source.  No reference counterpart (the reference resolves every scale).

constexpr int kSgsIn = 13, kSgsOut = 9;   // closure features and fluxes per point

// periodic image of any x or spanwise index on the unique points 2..n-1
__device__ __forceinline__ int wrap_any(int i, int n)
{
    if (i >= 2 && i <= n - 1) return i;
    const int m = n - 2;
    if (i >= 2 - m && i < 2) return i + m;
    if (i > n - 1 && i <= n - 1 + m) return i - m;
    int r = (i - 2) % m;
    if (r < 0) r += m;
    return r + 2;
}

// primitives (rho, u, v, w, T) at (i, j, k): the wall-plane ring on the
// walls, the conservative state elsewhere (exact divisions)
__device__ __forceinline__ void prim_at(const KParams &P, const double *q, int i, int j, int k, double x[5])
{
    i = wrap_any(i, P.n1);
    j = wrap_any(j, P.n2);
    if (k <= 1 || k >= P.n3) {
        const double *W = P.wp + (size_t)(k <= 1 ? 0 : 8) * P.plane + (long long)j * P.px + i;
        x[0] = W[0]; x[1] = W[P.plane]; x[2] = W[2 * P.plane]; x[3] = W[3 * P.plane]; x[4] = W[5 * P.plane];
        return;
    }
    const long long o = (long long)k * P.plane + (long long)j * P.px + i;
    const double r = q[o], ri = 1.0 / r;
    x[0] = r;
    x[1] = q[P.vol + o] * ri;
    x[2] = q[2 * P.vol + o] * ri;
    x[3] = q[3 * P.vol + o] * ri;
    x[4] = q[4 * P.vol + o] * ri - P.ggMh * ((x[1] * x[1] + x[2] * x[2]) + x[3] * x[3]);
}

// Favre-filtered (rho, u, v, w, T) at (i, j, k): a box of width fw (even)
// in x and spanwise, the trapezoid weights (1/2, 1, .., 1, 1/2) / fw per
// direction; fw = 0 returns the point's own values.  With prod != 0 it also
// returns the filtered rho*u_a*u_b (uu, vv, ww, uv, uw, vw) and rho*u_b*T.
__device__ __forceinline__ void favre_at(const KParams &P, const double *q, int i, int j, int k, int fw,
                                         double f[5], double *prod)
{
    if (fw == 0) {
        prim_at(P, q, i, j, k, f);
        if (prod) {
            const double r = f[0], u = f[1], v = f[2], w = f[3], T = f[4];
            prod[0] = r * u * u; prod[1] = r * v * v; prod[2] = r * w * w;
            prod[3] = r * u * v; prod[4] = r * u * w; prod[5] = r * v * w;
            prod[6] = r * u * T; prod[7] = r * v * T; prod[8] = r * w * T;
        }
        return;
    }
    const int h = fw / 2;
    double sr = 0, su = 0, sv = 0, sw = 0, sT = 0, sp[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = -h; b <= h; b++) {
        const double wb = (b == -h || b == h) ? 0.5 : 1.0;
        for (int a = -h; a <= h; a++) {
            const double wgt = wb * ((a == -h || a == h) ? 0.5 : 1.0);
            double x[5];
            prim_at(P, q, i + a, j + b, k, x);
            const double r = x[0], u = x[1], v = x[2], w = x[3], T = x[4], rw = wgt * r;
            sr += wgt * r; su += rw * u; sv += rw * v; sw += rw * w; sT += rw * T;
            if (prod) {
                sp[0] += rw * u * u; sp[1] += rw * v * v; sp[2] += rw * w * w;
                sp[3] += rw * u * v; sp[4] += rw * u * w; sp[5] += rw * v * w;
                sp[6] += rw * u * T; sp[7] += rw * v * T; sp[8] += rw * w * T;
            }
        }
    }
    const double nrm = 1.0 / ((double)fw * (double)fw);
    f[0] = sr * nrm;
    f[1] = su / sr; f[2] = sv / sr; f[3] = sw / sr; f[4] = sT / sr;
    if (prod)
        for (int c = 0; c < 9; c++) prod[c] = sp[c] * nrm;
}

struct SgsSampling {
    int sx, sy, sz, fw;          // gradient strides, filter width
    int i0, ni, j0, nj, k0, nk;  // sample points i0 + sx*a (a < ni), j0 + sy*b, k0 + sz*c
    const double *x3;            // x3(1..nP3) at x3[k-1]
    float *X, *T;                // [n][13], [n][9] (T may be null)
    bool soa;                    // X as [13][n] instead (the closure run's layout)
};

// Features (and with T the filtered subgrid fluxes) at every sample point.
// Gradients by central differences of the filtered fields at the sample
// strides (the coarse grid's spacing); y+ from the wall shear of the last
// statistics step.
__global__ void k_sgs_sample(const KParams P, const double *q, const SgsSampling S)
{
    const long long n = (long long)S.ni * S.nj * S.nk;
    const double Lx = 1.0 / P.invdx, Ly = 1.0 / P.invdy;   // dx, dy
    const int n3 = P.n3;
    const double tw = 0.5 * (P.stat[23 * n3] - P.stat[23 * n3 + 1]);
    const double rw = 0.5 * (P.stat[0] + P.stat[n3 - 1]);
    // before the first statistics step the sums are zero: y+ is then 0
    const double ut = rw > 0.0 ? sqrt(fmax(tw, 0.0) / rw) : 0.0, muw = 0.5 * (P.muwb + P.muwt);
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(s % S.ni), b = (int)((s / S.ni) % S.nj), c = (int)(s / ((long long)S.ni * S.nj));
        const int i = S.i0 + S.sx * a, j = S.j0 + S.sy * b, k = S.k0 + S.sz * c;
        double f0[5], prod[9], fxp[5], fxm[5], fyp[5], fym[5], fzp[5], fzm[5];
        favre_at(P, q, i, j, k, S.fw, f0, S.T ? prod : nullptr);
        favre_at(P, q, i + S.sx, j, k, S.fw, fxp, nullptr);
        favre_at(P, q, i - S.sx, j, k, S.fw, fxm, nullptr);
        favre_at(P, q, i, j + S.sy, k, S.fw, fyp, nullptr);
        favre_at(P, q, i, j - S.sy, k, S.fw, fym, nullptr);
        const int kp = min(k + S.sz, n3), km = max(k - S.sz, 1);
        favre_at(P, q, i, j, kp, S.fw, fzp, nullptr);
        favre_at(P, q, i, j, km, S.fw, fzm, nullptr);
        const double cx = 1.0 / (2.0 * S.sx * Lx), cy = 1.0 / (2.0 * S.sy * Ly);
        const double cz = 1.0 / (S.x3[kp - 1] - S.x3[km - 1]);
        float *X = S.soa ? S.X + s : S.X + s * 13;
        const long long xc = S.soa ? n : 1;
        // du_a/dx_b, a = u, v, w (fields 1..3), b = x, spanwise, wall-normal; then dT/dx_b
        for (int m = 0; m < 4; m++) {
            X[(3 * m + 0) * xc] = (float)((fxp[m + 1] - fxm[m + 1]) * cx);
            X[(3 * m + 1) * xc] = (float)((fyp[m + 1] - fym[m + 1]) * cy);
            X[(3 * m + 2) * xc] = (float)((fzp[m + 1] - fzm[m + 1]) * cz);
        }
        const double d = fmin(S.x3[k - 1] - S.x3[0], S.x3[n3 - 1] - S.x3[k - 1]);
        X[12 * xc] = (float)(rw * ut * d * (1.0 / P.invRe) / muw);
        if (S.T) {
            const double r = f0[0], u = f0[1], v = f0[2], w = f0[3], T = f0[4];
            float *Tg = S.T + s * 9;
            Tg[0] = (float)(prod[0] - r * u * u);
            Tg[1] = (float)(prod[1] - r * v * v);
            Tg[2] = (float)(prod[2] - r * w * w);
            Tg[3] = (float)(prod[3] - r * u * v);
            Tg[4] = (float)(prod[4] - r * u * w);
            Tg[5] = (float)(prod[5] - r * v * w);
            Tg[6] = (float)(prod[6] - r * u * T);
            Tg[7] = (float)(prod[7] - r * v * T);
            Tg[8] = (float)(prod[8] - r * w * T);
        }
    }
}

// Closure source at the interior points from the subgrid fluxes Y [9][n]
// (n = (n1-2)(n2-2)(n3-2), index ((k-2)(n2-2) + (j-2))(n1-2) + i-2; zero on
// the walls): S(rho u_a) = -d tau_ab / dx_b, S(rho E) = -gama d q_b / dx_b
// (the enthalpy flux gama*rho*u*T of the reference's energy equation).
__global__ void k_sgs_div(const KParams P, const float *Y, double gama, double *S)
{
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3, m1 = n1 - 2, m2 = n2 - 2;
    const long long n = (long long)m1 * m2 * (n3 - 2);
    auto at = [&](int i, int j, int k, int c) -> double {
        if (k <= 1 || k >= n3) return 0.0;
        i = wrap_any(i, n1);
        j = wrap_any(j, n2);
        return (double)Y[(long long)c * n + (((long long)(k - 2) * m2) + (j - 2)) * m1 + (i - 2)];
    };
    // flux component of (row a, direction b): tau_ab, or q_b for the energy row
    auto comp = [](int a, int b) {
        const int t[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
        return a < 3 ? t[a][b] : 6 + b;
    };
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const int i = 2 + (int)(s % m1), j = 2 + (int)((s / m1) % m2), k = 2 + (int)(s / ((long long)m1 * m2));
        const double cz = P.czh[k];
        for (int a = 0; a < 4; a++) {
            const double d = (at(i + 1, j, k, comp(a, 0)) - at(i - 1, j, k, comp(a, 0))) * P.hdx +
                             (at(i, j + 1, k, comp(a, 1)) - at(i, j - 1, k, comp(a, 1))) * P.hdy +
                             (at(i, j, k + 1, comp(a, 2)) - at(i, j, k - 1, comp(a, 2))) * cz;
            S[(size_t)a * n + s] = a < 3 ? -d : -gama * d;
        }
    }
}

// q_out += cdt * S at every stored point of the interior planes (periodic
// duplicates and ghosts take their image's source)
__global__ void k_sgs_apply(const KParams P, double *qo, const double *S, double cdt)
{
    const int n1 = P.n1, n2 = P.n2, n3 = P.n3, m1 = n1 - 2, m2 = n2 - 2;
    const long long n = (long long)m1 * m2 * (n3 - 2);
    const long long tot = (long long)(n1 + 2) * (n2 + 2) * (n3 - 2);
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < tot; s += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(s % (n1 + 2)), j = (int)((s / (n1 + 2)) % (n2 + 2)), k = 2 + (int)(s / ((long long)(n1 + 2) * (n2 + 2)));
        const int iu = wrap_any(i, n1), ju = wrap_any(j, n2);
        const long long src = (((long long)(k - 2) * m2) + (ju - 2)) * m1 + (iu - 2);
        const long long o = (long long)k * P.plane + (long long)j * P.px + i;
        // S rows: rho*u, rho*v, rho*w, rho*E (state variables 1..4)
#pragma unroll
        for (int a = 0; a < 4; a++) qo[o + (a + 1) * P.vol] += cdt * S[(size_t)a * n + src];
    }
}

// start of a step in a graph replay: step += 1, time += dt (the host's order)
__global__ void k_clock_advance(DevClock *clk, double dt)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        clk->step = clk->step + 1;
        clk->time = clk->time + dt;
    }
}

// double -> float copy (seeds the mixed-precision stage buffers)
__global__ void k_to_float(const double *a, float *b, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// self-test of pow07 against the CUDA math library's pow (diagnostics only)
__global__ void k_selftest_pow07(const double *T, double *mine, double *libm, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        mine[i] = pow07(T[i]);
        libm[i] = pow(T[i], 0.7);
    }
}

// ---------------------------------------------------------------------------
// Persistent ensemble kernel.
//
// One launch runs a block of L time steps of every member of an ensemble.  The
// host lays the work out as phases -- for each member and step: the clock
// advance, then per RK stage the stage kernel's CTAs and the wall kernel's
// blocks, then on statistics steps the two statistics passes -- each phase a
// number of units (one unit = one CTA's work of the kernel it replaces), and
// lists all units of all members in one work list, members interleaved phase
// by phase.  CTAs take units from the list in order through an atomic
// counter.  A unit may start once its member has completed every unit of its
// earlier phases: the member's completion counter reaches the phase's `need`.
// Units are taken in list order and a unit only waits for units earlier in the
// list, which running CTAs hold, so the launch always progresses; each wait is
// still bounded (about a second), after which the CTA records the error and
// stops.
// Every member's arithmetic is the stand-alone kernels' code, so its results
// are bit for bit those of chan_step.
enum PKind { kPClock = 0, kPStage = 1, kPWall = 2, kPStatsPart = 3, kPStatsFin = 4 };

struct PPhase {
    int member;
    int kind;            // PKind
    int variant;         // stage: 0 FP64, 1..3 mixed first / middle / last; wall: 0 double, 1 float state
    int tile;            // stage: CHAN_TILE_32x8 (0) or CHAN_TILE_16x16 (2)
    int nx, ny;          // stage: tiles in x, y; wall: blocks in x, y; stats: blocks per plane (S)
    int kp;              // index of the member's KParams record for this phase
    int units;
    int group;           // wall: wall blocks per unit (the blocks are short)
    unsigned long long need;    // member's completed units before this phase may start
    double dt;                  // clock advance
    const CUtensorMap *tm;      // stage: tensor map of the input buffer
    const CUtensorMap *tmb;     // stage: tensor map of the RK base (tiles that stage it by bulk copy)
    const double *q;            // statistics: the state buffer
    double *part;               // statistics: partial sums
};

struct PItem {
    int phase;
    int unit;
};

// The members' parameter records of the running persistent block, in constant
// memory: a stage body reads its record's fields many times, and from the
// constant cache those reads are cheap where global memory would put a load
// and its latency on each.  A block's graph copies its records here first.
constexpr int kEnsKps = 64;
__constant__ KParams c_ens_kps[kEnsKps];

struct PPlan {
    const PPhase *phases;
    const PItem *items;         // the work list: members' units interleaved phase by phase
    long long nitems;
    unsigned long long *done;   // [members] completed units
    unsigned long long *next;   // work-list position
    int *err;                   // 1: a dependency wait gave up
    DevClock *clk;              // [members]
#ifdef CHAN_PERSIST_GLOBAL_KPS
    const KParams *kps;
#endif
};

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

constexpr unsigned long long kDepWaitNs = 1000000000ull;

template <int TI, int TJ, typename QI, typename QO, typename R>
__device__ __forceinline__ void pstage(const PPhase &F, const KParams &P, int unit, int tid, unsigned char *smem)
{
    const int bx = unit % F.nx, r = unit / F.nx, by = r % F.ny, bz = r / F.ny;
    stage_body<TI, TJ, QI, QO, R, 2, true>(P, F.tm, F.tmb, bx, by, bz, tid % TI, tid / TI, smem);
}

#ifndef CHAN_PMINB_MIXED
#define CHAN_PMINB_MIXED 2   // resident CTAs per SM of the mixed-precision persistent kernel (3 spills ~1.3 KB per thread)
#endif
template <bool MIXED>
struct PersistShape {
    // dynamic shared memory: the largest unit's, plus the work-item slot
    static constexpr size_t st = MIXED ? (StageShape<32, 8, float>::bytes > StageShape<16, 16, float>::bytes
                                               ? StageShape<32, 8, float>::bytes
                                               : StageShape<16, 16, float>::bytes)
                                       : (StageShape<32, 8, double>::bytes > StageShape<16, 16, double>::bytes
                                              ? StageShape<32, 8, double>::bytes
                                              : StageShape<16, 16, double>::bytes);
    static constexpr size_t wall = sizeof(double) * 2 * 6 * kWallHY * kWallHX;
    static constexpr size_t body = ((st > wall ? st : wall) + 127) / 128 * 128;
    static constexpr size_t bytes = body + 128;
    static constexpr int minb = MIXED ? CHAN_PMINB_MIXED : 2;
};

template <bool MIXED>
__global__ void __launch_bounds__(256, PersistShape<MIXED>::minb) k_ensemble(const PPlan plan)
{
    using PS = PersistShape<MIXED>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    long long *s_item = reinterpret_cast<long long *>(smem_raw + PS::body);
    int *s_ok = reinterpret_cast<int *>(s_item + 1);
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) {
            // the next unit of the work list; wait (bounded) until its member has
            // completed the units of its earlier phases
            long long it = (long long)atomicAdd(plan.next, 1ull);
            if (it < plan.nitems && *(volatile int *)plan.err) it = plan.nitems;   // after an error: stop
            int ok = 1;
            if (it < plan.nitems) {
                const PPhase &F = plan.phases[plan.items[it].phase];
                const unsigned long long *d = plan.done + F.member;
                if (ld_acquire_u64(d) < F.need) {
                    const unsigned long long t0 = global_ns();
                    while (ld_acquire_u64(d) < F.need) {
                        if (global_ns() - t0 > kDepWaitNs) { ok = 0; break; }
                        __nanosleep(256);
                    }
                }
                if (!ok) atomicExch(plan.err, 1);
            }
            *s_item = it;
            *s_ok = ok;
        }
        __syncthreads();
        const long long it = *s_item;
        const int ok = *s_ok;
        __syncthreads();
        if (it >= plan.nitems || !ok) break;
        const PItem I = plan.items[it];
        const PPhase &F = plan.phases[I.phase];
#ifdef CHAN_PERSIST_GLOBAL_KPS
        const KParams &P = plan.kps[F.kp];   // measurement variant: records in global memory
#else
        const KParams &P = c_ens_kps[F.kp];
#endif
        switch (F.kind) {
        case kPClock:
            if (tid == 0) {
                DevClock *c = plan.clk + F.member;
                c->step = c->step + 1;
                c->time = c->time + F.dt;
            }
            break;
        case kPStage:
            if (!MIXED) {
                if (F.tile == 0) pstage<32, 8, double, double, double>(F, P, I.unit, tid, smem_raw);
                else pstage<16, 16, double, double, double>(F, P, I.unit, tid, smem_raw);
            } else if (F.tile == 0) {
                if (F.variant == 1) pstage<32, 8, double, float, float>(F, P, I.unit, tid, smem_raw);
                else if (F.variant == 2) pstage<32, 8, float, float, float>(F, P, I.unit, tid, smem_raw);
                else pstage<32, 8, float, double, float>(F, P, I.unit, tid, smem_raw);
            } else {
                if (F.variant == 1) pstage<16, 16, double, float, float>(F, P, I.unit, tid, smem_raw);
                else if (F.variant == 2) pstage<16, 16, float, float, float>(F, P, I.unit, tid, smem_raw);
                else pstage<16, 16, float, double, float>(F, P, I.unit, tid, smem_raw);
            }
            break;
        case kPWall: {
            WallStage &sp = *reinterpret_cast<WallStage *>(smem_raw);
            const int nb = F.nx * F.ny * 2, b0 = I.unit * F.group, b1 = min(b0 + F.group, nb);
            for (int b = b0; b < b1; b++) {
                if (b > b0) __syncthreads();   // the staging area is reused
                const int bx = b % F.nx, r = b / F.nx, by = r % F.ny, wall = r / F.ny;
                if (F.variant == 0) wall_body<double>(P, bx, by, wall, tid % kWallBX, tid / kWallBX, sp);
                else wall_body<float>(P, bx, by, wall, tid % kWallBX, tid / kWallBX, sp);
            }
            break;
        }
        case kPStatsPart:
            stats_part_body(P, F.q, 1, 1, F.nx, F.part, I.unit, tid, *reinterpret_cast<StatRed *>(smem_raw));
            break;
        case kPStatsFin: {
            const int pb = I.unit * 8 + (tid >> 5);
            if (pb < P.n3 + 2) stats_fin_body(P, 1, 1, F.nx, F.part, pb, tid & 31);
            break;
        }
        default:
            break;
        }
        // the unit's writes (all threads) before its completion is counted
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicAdd(plan.done + F.member, 1ull);
        }
    }
}

}  // namespace chan
