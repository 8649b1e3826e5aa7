// chanrhs.cu -- host side of the C ABI declared in include/chanrhs.h.
//
// The context owns every device buffer; host arrays are only read or
// written inside chan_upload, chan_download and chan_stats.  All work is
// queued on one CUDA stream per context.
#include "chanrhs.h"
#include "chan_internal.h"
#include "chan_kernels.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

// Stage-kernel tile shapes: TI columns in x (one warp row) by TJ rows in y.
// Each shape has the plain FP64 kernel and the three mixed-precision stage
// kernels, without and with the buoyancy term.
using StageFn = void (*)(const chan::KParams, const CUtensorMap, const CUtensorMap);
struct StageSet {
    int ti, tj;
    StageFn k[2][4];   // [buoyancy][0 FP64, 1 mixed first stage, 2 mixed middle, 3 mixed last]
    size_t smem, smemf;
};
template <int TI_, int TJ_, bool B>
void fill_stage_set(StageSet &s)
{
    s.k[B][0] = chan::k_stage<TI_, TJ_, double, double, double, B>;
    s.k[B][1] = chan::k_stage<TI_, TJ_, double, float, float, B>;
    s.k[B][2] = chan::k_stage<TI_, TJ_, float, float, float, B>;
    s.k[B][3] = chan::k_stage<TI_, TJ_, float, double, float, B>;
}
template <int TI_, int TJ_>
StageSet make_stage_set()
{
    StageSet s{};
    s.ti = TI_;
    s.tj = TJ_;
    fill_stage_set<TI_, TJ_, false>(s);
    fill_stage_set<TI_, TJ_, true>(s);
    s.smem = chan::StageShape<TI_, TJ_, double>::bytes;
    s.smemf = chan::StageShape<TI_, TJ_, float>::bytes;
    return s;
}
// CHAN_TILE_32x8 (default), CHAN_TILE_32x4, CHAN_TILE_16x16, CHAN_TILE_32x16
const StageSet kStageSets[CHAN_NTILES] = {make_stage_set<32, 8>(), make_stage_set<32, 4>(),
                                          make_stage_set<16, 16>(), make_stage_set<32, 16>()};
constexpr int kMaxSplit = 16;   // statistics blocks per plane, at most

std::string g_init_error;

struct ProfPair {
    int cls;
    cudaEvent_t a, b;
};

}  // namespace

struct chan_ctx {
    chan_params p{};
    int dev = 0;
    cudaStream_t stream = nullptr;
    chan::KParams kp{};
    double *q[3] = {nullptr, nullptr, nullptr};   // plain FP64: state and two stage buffers
    float *qf[2] = {nullptr, nullptr};            // mixed precision: the two stage buffers in float
    bool mixed = false;
    float *tabf = nullptr;                        // per-k tables in float (mixed)
    double *wp = nullptr, *cs = nullptr, *tabs = nullptr, *stat = nullptr, *dvar = nullptr, *tacc = nullptr;
    double *hwt = nullptr;   // hD of the top wall plane, staged inside a stage
    double *spart = nullptr; // statistics partial sums [(nP3+2)*nsplit][23]
    int nsplit = 1;          // blocks per plane in the statistics pass
    unsigned char *wmask[2] = {nullptr, nullptr};  // wall-BC plug-in arrays (allocated on first use)
    double *wuv[2] = {nullptr, nullptr}, *wx1[2] = {nullptr, nullptr};
    long long tavg_samples = 0;  // statistics steps summed into tacc since chan_time_avg_start
    double tavg_t0 = 0.0, tavg_t1 = 0.0;
    chan::DevStatus *status = nullptr;
    chan::DevStatus *h_status = nullptr;
    int n1 = 0, n2 = 0, n3 = 0, px = 0, NJ = 0;
    long long plane = 0, vol = 0;
    int tile = CHAN_TILE_32x8, ntx = 0, nty = 0, nchunks = 1, kchunk = 1;   // stage-kernel launch shape
    // tensor maps of the stage kernel's box copies, per tile shape: the three
    // FP64 state buffers, or the two float stage buffers (mixed precision)
    CUtensorMap tmd[CHAN_NTILES][3];
    CUtensorMap tmf[CHAN_NTILES][2];
    CUtensorMap tmb[CHAN_NTILES];   // the RK base (the FP64 step state) by tile: box TI x TJ x 1 x 5
    int nstage = 2;
    int cur = 0;             // buffer holding the latest state
    bool uploaded = false;
    long long nstep = 0;
    double time = 0.0;
    long long sync_nstep = 0;  // counters at the last status read without a blow-up
    double sync_time = 0.0;
    std::string err;
    bool prof = false;
    std::vector<ProfPair> prof_pairs;
    std::vector<cudaEvent_t> ev_pool;
    size_t dev_bytes = 0;
    std::vector<double> hx3;      // x3 given to chan_init
    struct Guarded {
        double *base;
        size_t n;
    };
    std::vector<Guarded> guarded;  // guard-zoned state buffers (dalloc)
    // diagnostics series (allocated by chan_diag_enable)
    int diag_every = 0, diag_cap = 0, diag_reclen = 0;
    long long diag_count = 0;     // records written since the last chan_diag_read
    double *diag_rec = nullptr, *diag_part = nullptr, *diag_x3 = nullptr;
    chan::DiagParams dp{};
    // fluctuation / Q-criterion buffers (allocated on first use)
    double *dq = nullptr, *dxyz = nullptr;
    // ensemble membership: the device clock its graph replays read, and a
    // counter of the kernel-visible settings, bumped by every call that
    // changes them, so that an ensemble knows when its captured graph is stale
    chan::DevClock *dclk = nullptr;
    long long epoch = 0;
    // learned subgrid closure (chan_set_closure): features, fluxes, source
    chan_closure *cl = nullptr;
    bool closure_on = false;
    bool closure_every_stage = false;   // else the source of a step's first stage is held for its other stages
    bool sgs_valid = false;             // sgsS holds a source for the current step
    double *dx3 = nullptr;                 // x3 on the device (allocated on first use)
    float *sgsX = nullptr, *sgsY = nullptr;
    double *sgsS = nullptr;
    int *sgsflag = nullptr;
};

namespace {

int fail(chan_ctx *c, const char *what, cudaError_t e)
{
    char buf[512];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    if (c) c->err = buf; else g_init_error = buf;
    return CHAN_ECUDA;
}

#define CK(c, call)                                   \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) return fail((c), #call, e_); \
    } while (0)

cudaEvent_t get_event(chan_ctx *c)
{
    if (!c->ev_pool.empty()) {
        cudaEvent_t e = c->ev_pool.back();
        c->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

// bracket a launch with events when profiling is on
struct ProfScope {
    chan_ctx *c;
    int cls;
    cudaEvent_t a = nullptr, b = nullptr;
    ProfScope(chan_ctx *c_, int cls_) : c(c_), cls(cls_)
    {
        if (c->prof) {
            a = get_event(c);
            b = get_event(c);
            if (a) cudaEventRecord(a, c->stream);
        }
    }
    ~ProfScope()
    {
        if (c->prof && a && b) {
            cudaEventRecord(b, c->stream);
            c->prof_pairs.push_back({cls, a, b});
        }
    }
};

// one-sided wall coefficients, v1.10/codes/main_v1.9.f90:59-83 (x3 1-based)
void wall_coeffs(const double *x3, int n3, double out[14])
{
    const double one = 1.0, haf = 0.5;
    double dz1 = x3[2] - x3[1];
    double alpha = (x3[3] - x3[2]) / dz1;
    double t = dz1 * alpha * (alpha + one);
    out[0] = (one - (alpha + one) * (alpha + one)) / t;
    out[1] = ((alpha + one) * (alpha + one)) / t;
    out[2] = -one / t;
    t = haf * (dz1 * dz1) * alpha * (alpha + one);
    out[3] = alpha / t;
    out[4] = -(alpha + one) / t;
    out[5] = one / t;
    double dzN = x3[n3] - x3[n3 - 1];
    alpha = (x3[n3 - 1] - x3[n3 - 2]) / dzN;
    t = dzN * alpha * (alpha + one);
    out[6] = ((alpha + one) * (alpha + one) - one) / t;
    out[7] = -((alpha + one) * (alpha + one)) / t;
    out[8] = one / t;
    t = haf * (dzN * dzN) * alpha * (alpha + one);
    out[9] = alpha / t;
    out[10] = -(alpha + one) / t;
    out[11] = one / t;
    out[12] = dz1;
    out[13] = dzN;
}

// cuTensorMapEncodeTiled from the driver, through the runtime (no -lcuda)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }
    return fn;
}

// tensor map of one state buffer [5][nP3+2][nP2+2][px] for the stage
// kernel's box copies: box (TI+4) x (TJ+4) x 1 plane x 5 variables, no
// swizzle, points beyond nP1+1 / nP2+1 read as zero.  A box's x origin is a
// multiple of TI (16 or 32 elements), so every copy starts on a 16-byte
// boundary; the rows, planes and variables are px, plane and vol elements
// apart (multiples of 8 elements).
int make_state_map(chan_ctx *c, CUtensorMap *m, void *base, bool is_float, int ti, int tj, int halo = 2)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) { c->err = "cuTensorMapEncodeTiled is not available"; return CHAN_ECUDA; }
    const cuuint64_t es = is_float ? 4 : 8;
    const cuuint64_t dims[4] = {(cuuint64_t)c->n1 + 2, (cuuint64_t)c->n2 + 2, (cuuint64_t)c->n3 + 2, 5};
    const cuuint64_t strides[3] = {(cuuint64_t)c->px * es, (cuuint64_t)c->plane * es, (cuuint64_t)c->vol * es};
    const cuuint32_t box[4] = {(cuuint32_t)(ti + 2 * halo), (cuuint32_t)(tj + 2 * halo), 1, 5};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = enc(m, is_float ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base,
                           dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        c->err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        return CHAN_ECUDA;
    }
    return CHAN_OK;
}

// the tensor map of the current stage's input buffer (any map when that
// stage loads its boxes with per-thread loads)
const CUtensorMap &stage_map(const chan_ctx *c)
{
    for (int b = 0; b < 3; b++)
        if (!c->mixed && c->kp.qin == (const void *)c->q[b]) return c->tmd[c->tile][b];
    for (int b = 0; b < 2; b++)
        if (c->mixed && c->kp.qin == (const void *)c->qf[b]) return c->tmf[c->tile][b];
    return c->tmd[c->tile][0];
}

void set_stage(chan_ctx *c, int iter)
{
    chan::KParams &k = c->kp;
    const double dt = c->p.dt;
    // stage buffers: B and C are q[1], q[2] (FP64) or qf[0], qf[1] (mixed precision)
    void *A = c->q[0];
    void *B = c->mixed ? (void *)c->qf[0] : (void *)c->q[1];
    void *Cb = c->mixed ? (void *)c->qf[1] : (void *)c->q[2];
    if (c->nstage == 3) {
        if (iter == 1) {
            k.qin = A; k.qbase = c->q[0]; k.qout = B;
            k.rk_mode = 0; k.rk_a = 0.0; k.rk_b = 1.0; k.rk_cdt = dt;
        } else if (iter == 2) {
            k.qin = B; k.qbase = c->q[0]; k.qout = Cb;
            k.rk_mode = 2; k.rk_a = 0.75; k.rk_b = 0.25; k.rk_cdt = 0.25 * dt;
        } else {
            k.qin = Cb; k.qbase = c->q[0]; k.qout = A;
            k.rk_mode = 2; k.rk_a = 1.0 / 3.0; k.rk_b = 2.0 / 3.0; k.rk_cdt = (2.0 / 3.0) * dt;
        }
    } else {
        if (iter == 1) {
            // solV(:,2)=solV(:,1); solV(:,1)+=haf*dt*R  (main_v1.9.f90:575-578)
            k.qin = A; k.qbase = c->q[0]; k.qout = B;
            k.rk_mode = 0; k.rk_a = 0.0; k.rk_b = 1.0; k.rk_cdt = 0.5 * dt;
        } else {
            // solV(:,1)=solV(:,2)+dt*R  (main_v1.9.f90:580-582)
            k.qin = B; k.qbase = c->q[0]; k.qout = A;
            k.rk_mode = 1; k.rk_a = 1.0; k.rk_b = 0.0; k.rk_cdt = dt;
        }
    }
}

// stage-kernel launch shape: tile shape and number of k-chunks (0: the
// chunk count whose CTAs fill whole waves of resident CTAs with the least
// prologue overhead per marched plane)
int set_launch(chan_ctx *c, int tile, int nchunks)
{
    if (tile < 0 || tile >= CHAN_NTILES) { c->err = "unknown tile shape"; return CHAN_EINVAL; }
    const StageSet &ss = kStageSets[tile];
    const int nz = c->n3 - 2;
    if (nchunks < 0 || nchunks > nz) { c->err = "k-chunk count out of range"; return CHAN_EINVAL; }
    const int ntx = (c->n1 - 2 + ss.ti - 1) / ss.ti, nty = (c->n2 - 2 + ss.tj - 1) / ss.tj;
    if (nchunks == 0) {
        int sms = 148, occ = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
        const int v = c->mixed ? 2 : 0;
        CK(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ss.k[0][v], ss.ti * ss.tj,
                                                            v == 0 ? ss.smem : ss.smemf));
        if (occ < 1) occ = 1;
        const long long slots = (long long)sms * occ, tiles = (long long)ntx * nty;
        double best = -1.0;
        for (int nc = 1; nc <= nz; nc++) {
            const int chunk = (nz + nc - 1) / nc;
            if ((nz + chunk - 1) / chunk != nc) continue;
            const long long ctas = tiles * nc;
            const long long waves = (ctas + slots - 1) / slots;
            const double eff = (double)ctas / (double)(waves * slots) * (double)chunk / (chunk + 2.5);
            if (eff > best + 1e-9) { best = eff; nchunks = nc; }
        }
    }
    // the chunk count that a chunk length of ceil(nz/nchunks) really gives
    const int chunk = (nz + nchunks - 1) / nchunks;
    c->tile = tile;
    c->ntx = ntx;
    c->nty = nty;
    c->kchunk = chunk;
    c->nchunks = (nz + chunk - 1) / chunk;
    c->kp.kchunk = chunk;
    c->epoch++;
    return CHAN_OK;
}

// device copy of x3 (closure features need the wall-normal coordinates)
int ensure_dx3(chan_ctx *c)
{
    if (c->dx3) return CHAN_OK;
    CK(c, cudaMalloc((void **)&c->dx3, (size_t)c->n3 * sizeof(double)));
    CK(c, cudaMemcpy(c->dx3, c->hx3.data(), (size_t)c->n3 * sizeof(double), cudaMemcpyHostToDevice));
    c->dev_bytes += (size_t)c->n3 * sizeof(double);
    return CHAN_OK;
}

// features of the stage input at every interior point, the closure MLP, and
// the source it gives (applied to the stage output after the stage kernel)
int closure_source(chan_ctx *c)
{
    chan::SgsSampling S{};
    S.sx = S.sy = S.sz = 1;
    S.fw = 0;
    S.i0 = 2; S.ni = c->n1 - 2;
    S.j0 = 2; S.nj = c->n2 - 2;
    S.k0 = 2; S.nk = c->n3 - 2;
    S.x3 = c->dx3;
    S.X = c->sgsX;
    S.T = nullptr;
    S.soa = true;
    const long long n = (long long)S.ni * S.nj * S.nk;
    chan::k_sgs_sample<<<1184, 128, 0, c->stream>>>(c->kp, (const double *)c->kp.qin, S);
    CK(c, cudaGetLastError());
    int r = chan_internal_infer(c->cl, c->sgsX, c->sgsY, n, true, c->stream, c->sgsflag);
    if (r) { c->err = "closure inference"; return r; }
    chan::k_sgs_div<<<1184, 256, 0, c->stream>>>(c->kp, c->sgsY, c->p.gama, c->sgsS);
    CK(c, cudaGetLastError());
    return CHAN_OK;
}

int launch_stage(chan_ctx *c, int iter, bool check, long long step, double time)
{
    set_stage(c, iter);
    c->kp.time = time;
    c->cur = c->kp.qout == (void *)c->q[0] ? 0 : (c->kp.qout == (void *)c->q[1] ? 1 : 2);
    c->kp.check = check ? 1 : 0;
    c->kp.step = step;
    const bool last = iter == c->nstage;
    if (c->closure_on && (iter == 1 || c->closure_every_stage || !c->sgs_valid)) {
        int r = closure_source(c);
        if (r) return r;
        c->sgs_valid = true;
    }
    {
        ProfScope ps(c, 0);
        const StageSet &ss = kStageSets[c->tile];
        dim3 grid(c->ntx, c->nty, c->nchunks), block(ss.ti, ss.tj);
        const int v = !c->mixed ? 0 : (iter == 1 ? 1 : (last ? 3 : 2));
        ss.k[c->kp.buoy_on ? 1 : 0][v]<<<grid, block, v == 0 ? ss.smem : ss.smemf, c->stream>>>(
            c->kp, stage_map(c), c->tmb[c->tile]);
    }
    if (c->closure_on) {
        chan::k_sgs_apply<<<1184, 256, 0, c->stream>>>(c->kp, (double *)c->kp.qout, c->sgsS, c->kp.rk_cdt);
        CK(c, cudaGetLastError());
    }
    CK(c, cudaGetLastError());
    {
        ProfScope ps(c, 1);
        dim3 block(32, 8), grid((c->n1 + 2 + 31) / 32, (c->n2 + 2 + 7) / 8, 2);
        if (c->mixed && !last)
            chan::k_wall<float><<<grid, block, 0, c->stream>>>(c->kp);
        else
            chan::k_wall<double><<<grid, block, 0, c->stream>>>(c->kp);
    }
    CK(c, cudaGetLastError());
    return CHAN_OK;
}

// mixed precision: the float stage buffers start as copies of the state, so
// their wall planes and wall ghosts (which no stage writes) hold the state's
int seed_float_stages(chan_ctx *c)
{
    if (!c->mixed) return CHAN_OK;
    const long long n = 5 * c->vol;
    for (int b = 0; b < 2; b++) {
        chan::k_to_float<<<1184, 256, 0, c->stream>>>(c->q[0], c->qf[b], n);
        CK(c, cudaGetLastError());
    }
    return CHAN_OK;
}

int launch_stats(chan_ctx *c, long long step, int moments, int tau)
{
    c->kp.step = step;
    ProfScope ps(c, 2);
    chan::k_stats_part<<<(c->n3 + 2) * c->nsplit, chan::kStatThreads, 0, c->stream>>>(c->kp, c->q[c->cur], moments,
                                                                                     tau, c->nsplit, c->spart);
    CK(c, cudaGetLastError());
    chan::k_stats_fin<<<c->n3 + 2, 32, 0, c->stream>>>(c->kp, moments, tau, c->nsplit, c->spart);
    CK(c, cudaGetLastError());
    return CHAN_OK;
}

int launch_diag(chan_ctx *c, long long step, double time)
{
    c->kp.step = step;
    double *rec = c->diag_rec + (size_t)(c->diag_count % c->diag_cap) * c->diag_reclen;
    chan::k_diag_ke<<<c->n3, chan::kStatThreads, 0, c->stream>>>(c->kp, c->q[c->cur], c->dp);
    CK(c, cudaGetLastError());
    chan::k_diag_fin<<<1 + 3 * c->dp.nplanes, chan::kStatThreads, 0, c->stream>>>(c->kp, c->q[c->cur], c->dp, rec,
                                                                                   time);
    CK(c, cudaGetLastError());
    c->diag_count++;
    return CHAN_OK;
}

// queue nsteps steps; host counters advance optimistically.  kCapture also
// advances the device clock at the start of every step (for a graph whose
// kernels read it); kCountOnly advances the host counters alone (after a
// graph replay did the work).
enum StepMode { kLaunch = 0, kCapture = 1, kCountOnly = 2 };
int enqueue_steps(chan_ctx *c, int nsteps, int mode = kLaunch)
{
    for (int s = 0; s < nsteps; s++) {
        const long long step = c->nstep + 1;
        if (mode == kCapture) {
            chan::k_clock_advance<<<1, 32, 0, c->stream>>>(c->dclk, c->p.dt);
            CK(c, cudaGetLastError());
        }
        if (mode != kCountOnly)
            for (int it = 1; it <= c->nstage; it++) {
                int r = launch_stage(c, it, it == c->nstage, step, c->time + c->p.dt);
                if (r) return r;
            }
        c->nstep = step;
        c->time = c->time + c->p.dt;
        if (mode != kCountOnly && c->diag_every > 0 && step % c->diag_every == 0) {
            int r = launch_diag(c, step, c->time);
            if (r) return r;
        }
        if (c->p.istat > 0 && step % c->p.istat == 0) {
            if (mode != kCountOnly) {
                int r = launch_stats(c, step, 1, 1);
                if (r) return r;
            }
            if (c->kp.acc_on) {
                if (c->tavg_samples == 0) c->tavg_t0 = c->time;
                c->tavg_t1 = c->time;
                c->tavg_samples++;
            }
        }
    }
    return CHAN_OK;
}

// read the device status; resolve the step/time of a blow-up
int read_status(chan_ctx *c, int32_t *ijk)
{
    CK(c, cudaMemcpyAsync(c->h_status, c->status, sizeof(chan::DevStatus), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    const chan::DevStatus &s = *c->h_status;
    if (s.blown) {
        if (s.blown_step < c->nstep && s.blown_step > c->sync_nstep) {
            // counters of the step that blew up, accumulated as the time loop does
            double t = c->sync_time;
            for (long long n = c->sync_nstep; n < s.blown_step; n++) t = t + c->p.dt;
            c->time = t;
            c->nstep = s.blown_step;
        }
        if (ijk) { ijk[0] = s.ijk[0]; ijk[1] = s.ijk[1]; ijk[2] = s.ijk[2]; }
        return CHAN_BLOWUP;
    }
    if (s.nonfinite) {
        if (ijk) { ijk[0] = s.nf_ijk[0]; ijk[1] = s.nf_ijk[1]; ijk[2] = s.nf_ijk[2]; }
        return CHAN_NONFINITE;
    }
    if (s.stall) {
        c->err = s.stall == 1 ? "stage kernel: a bulk box copy did not complete within its time limit"
                              : "stage kernel: shared-memory staging area not 128-byte aligned";
        return CHAN_ECUDA;
    }
    if (ijk) ijk[0] = ijk[1] = ijk[2] = 0;
    c->sync_nstep = c->nstep;
    c->sync_time = c->time;
    return CHAN_OK;
}

// Every state buffer sits between two guard zones of kGuard words holding
// kCanary (a NaN bit pattern no kernel writes).  chan_debug_canaries reads
// them back: any change means a kernel wrote outside its buffer.
constexpr size_t kGuard = 64;   // 512 bytes: the payload keeps 256-byte alignment
constexpr unsigned long long kCanary = 0x7ff4deadbeef0001ULL;

int dalloc(chan_ctx *c, double **p, size_t n)
{
    double *base = nullptr;
    cudaError_t e = cudaMalloc((void **)&base, (n + 2 * kGuard) * sizeof(double));
    if (e != cudaSuccess) {
        fail(c, "cudaMalloc", e);
        return CHAN_ENOMEM;
    }
    c->guarded.push_back({base, n});
    c->dev_bytes += (n + 2 * kGuard) * sizeof(double);
    *p = base + kGuard;
    std::vector<unsigned long long> pat(kGuard, kCanary);
    e = cudaMemcpyAsync(base, pat.data(), kGuard * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(base + kGuard + n, pat.data(), kGuard * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);   // pat is a host temporary
    if (e != cudaSuccess) return fail(c, "guard fill", e);
    e = cudaMemsetAsync(*p, 0, n * sizeof(double), c->stream);
    if (e != cudaSuccess) return fail(c, "cudaMemsetAsync", e);
    return CHAN_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free plane moments.
//
// Fortran post-processing programs of the reference (avg_v1.7.f90, fluc.f90)
// bind through iso_c_binding and have no way to call cudaMalloc or to keep a
// solver context, so they cannot supply device buffers.  chan_avg_spatial_noalloc
// serves them from one file-scope device array of fixed size.  Every GPU that
// loads this library holds the array until the process exits.
//
// Layout of the array per call: [23*nP3 results][7*nk*nP1*nP2 staged slab].
// Calls share the array and it keeps the last call's contents; calls that
// overlap on the GPU (two host threads, or two streams) race on it.
static __device__ __align__(256) double g_noalloc_scratch[CHAN_NOALLOC_MAX_DOUBLES];

// device address of g_noalloc_scratch in the current device's context.  It is
// looked up on every call (cudaGetSymbolAddress allocates nothing): an address
// kept from an earlier call would go stale if the context were reset and
// re-created in between.
double *noalloc_scratch()
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
        g_init_error = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
        return nullptr;
    }
    return (double *)p;
}

// blocks per plane of the statistics pass: about 16 blocks per SM, at least
// 4 point strides per block, at most kMaxSplit
int stats_split(int sms, int n1, int n2, int n3)
{
    const long long np = (long long)n1 * n2;
    int ns = (int)((16LL * sms + (n3 + 2) - 1) / (n3 + 2));
    const int cap = (int)std::max<long long>(1, np / (4LL * chan::kStatThreads));
    ns = std::min(std::min(ns, cap), kMaxSplit);
    return std::max(ns, 1);
}

// plane moments of a staged slab of var planes k0..k0+nk-1, in the reduction
// order of k_stats_part + k_stats_fin with S blocks per plane (so both paths
// give the same bits): S partial sums in turn, then their ordered sum
__global__ void __launch_bounds__(chan::kStatThreads) k_moments_slab(const double *slab, int n1, int n2, int nk,
                                                                     int k0, int n3, int S, double *res)
{
    __shared__ double red[chan::kStatThreads / 32][23];
    __shared__ double tot[23];
    const int kk = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long pl = (long long)n1 * n2;
    if (tid < 23) tot[tid] = 0.0;
    for (int sub = 0; sub < S; sub++) {
        double acc[23];
#pragma unroll
        for (int c = 0; c < 23; c++) acc[c] = 0.0;
        for (long long p = (long long)sub * chan::kStatThreads + tid; p < pl; p += (long long)S * chan::kStatThreads) {
            double x[7];
#pragma unroll
            for (int m = 0; m < 7; m++) x[m] = slab[((long long)m * nk + kk) * pl + p];
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
            const double sum = chan::warp_sum(acc[c]);
            if (lane == 0) red[warp][c] = sum;
        }
        __syncthreads();
        if (tid < 23) {
            double sum = 0.0;
            for (int w = 0; w < chan::kStatThreads / 32; w++) sum += red[w][tid];
            tot[tid] += sum;
        }
        __syncthreads();
    }
    if (tid < 23) res[(long long)tid * n3 + k0 + kk] = tot[tid] / (double)(n1 * n2);
}

}  // namespace

extern "C" {

const char *chan_version(void) { return "compchan3dmpi_b200 0.1 (sm_100a, fp64)"; }

const char *chan_last_error(chan_ctx *c)
{
    if (!c) return g_init_error.c_str();
    return c->err.c_str();
}

int chan_init(const chan_params *p, const double *x3, const double *jac, const double *invJac, chan_ctx **out)
{
    g_init_error.clear();
    if (!out) { g_init_error = "out is NULL"; return CHAN_EINVAL; }
    *out = nullptr;
    if (!p || !x3 || !jac || !invJac) { g_init_error = "NULL argument"; return CHAN_EINVAL; }
    if (p->nP[0] < 6 || p->nP[1] < 6 || p->nP[2] < 6) { g_init_error = "every nP must be >= 6"; return CHAN_EINVAL; }
    if ((long long)p->nP[0] * p->nP[1] * p->nP[2] > (1LL << 31)) { g_init_error = "grid too large"; return CHAN_EINVAL; }
    if (!(p->Re > 0) || !(p->Mac > 0) || !(p->dt > 0) || !(p->Pr > 0) || !(p->gama > 1)) {
        g_init_error = "Re, Mac, dt, Pr must be > 0 and gama > 1";
        return CHAN_EINVAL;
    }
    if (p->rk_scheme != CHAN_RK2 && p->rk_scheme != CHAN_RK3) { g_init_error = "rk_scheme must be 2 or 3"; return CHAN_EINVAL; }
    if (p->forcing != CHAN_FORCE_WALLSHEAR && p->forcing != CHAN_FORCE_NONE) { g_init_error = "bad forcing"; return CHAN_EINVAL; }
    if ((p->flags & ~CHAN_MIXED) != 0) { g_init_error = "flags must be 0 or CHAN_MIXED"; return CHAN_EINVAL; }
    if (p->istat < 0) { g_init_error = "istat must be >= 0"; return CHAN_EINVAL; }
    for (int k = 1; k < p->nP[2]; k++)
        if (!(x3[k] > x3[k - 1])) { g_init_error = "x3 must increase"; return CHAN_EINVAL; }

    chan_ctx *c = new chan_ctx();
    c->p = *p;
    c->dev = p->device;
    cudaError_t e = cudaSetDevice(c->dev);
    if (e != cudaSuccess) { fail(nullptr, "cudaSetDevice", e); delete c; return CHAN_ECUDA; }
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { fail(nullptr, "cudaStreamCreate", e); delete c; return CHAN_ECUDA; }

    const int n1 = p->nP[0], n2 = p->nP[1], n3 = p->nP[2];
    c->n1 = n1; c->n2 = n2; c->n3 = n3;
    c->px = ((n1 + 2) + 7) / 8 * 8;
    c->NJ = n2 + 2;
    c->plane = (long long)c->px * c->NJ;
    c->vol = c->plane * (n3 + 2);
    c->nstage = p->rk_scheme == CHAN_RK3 ? 3 : 2;
    c->hx3.assign(x3, x3 + n3);

    c->mixed = (p->flags & CHAN_MIXED) != 0;
    int r;
    for (int b = 0; b < (c->mixed ? 1 : 3); b++)
        if ((r = dalloc(c, &c->q[b], 5 * (size_t)c->vol))) { g_init_error = c->err; chan_free(c); return r; }
    if (c->mixed) {
        for (int b = 0; b < 2; b++) {
            double *t = nullptr;
            if ((r = dalloc(c, &t, (5 * (size_t)c->vol + 1) / 2))) { g_init_error = c->err; chan_free(c); return r; }
            c->qf[b] = reinterpret_cast<float *>(t);
        }
        double *t = nullptr;
        if ((r = dalloc(c, &t, (4 * (size_t)(n3 + 2) + 1) / 2))) { g_init_error = c->err; chan_free(c); return r; }
        c->tabf = reinterpret_cast<float *>(t);
    }
    if ((r = dalloc(c, &c->wp, 2 * 8 * (size_t)c->plane)) || (r = dalloc(c, &c->cs, (size_t)(n3 + 2) * 28)) ||
        (r = dalloc(c, &c->tabs, 4 * (size_t)(n3 + 2))) || (r = dalloc(c, &c->stat, 23 * (size_t)n3 + 2)) ||
        (r = dalloc(c, &c->tacc, 23 * (size_t)n3 + 2)) || (r = dalloc(c, &c->hwt, 4 * (size_t)c->plane)) ||
        (r = dalloc(c, &c->spart, 23 * (size_t)(n3 + 2) * kMaxSplit)) ||
        (r = dalloc(c, &c->dvar, 7 * (size_t)n1 * n2 * n3))) {
        g_init_error = c->err;
        chan_free(c);
        return r;
    }
    e = cudaMalloc((void **)&c->status, sizeof(chan::DevStatus));
    if (e == cudaSuccess) e = cudaMemsetAsync(c->status, 0, sizeof(chan::DevStatus), c->stream);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_status, sizeof(chan::DevStatus));
    if (e != cudaSuccess) { fail(nullptr, "status allocation", e); chan_free(c); return CHAN_ENOMEM; }

    // mesh-derived tables (1-based k stored at index k)
    std::vector<double> X3(n3 + 1), JAC(n3 + 1), INV(n3 + 1);
    for (int k = 1; k <= n3; k++) { X3[k] = x3[k - 1]; JAC[k] = jac[k - 1]; INV[k] = invJac[k - 1]; }
    double co[14];
    wall_coeffs(X3.data(), n3, co);

    const double Re = p->Re, Mac = p->Mac, gama = p->gama;
    const double dx = p->Lx / (double)(n1 - 1), dy = p->Ly / (double)(n2 - 1), dXi = 2.0 / (double)(n3 - 1);
    const double invdx = 1.0 / dx, invdy = 1.0 / dy, invdXi = 1.0 / dXi;
    std::vector<double> tab(4 * (size_t)(n3 + 2), 0.0);
    for (int k = 1; k <= n3; k++) {
        tab[0 * (n3 + 2) + k] = 0.5 * invdXi * INV[k];
        tab[1 * (n3 + 2) + k] = (invdXi * INV[k]) / 8.0;
        tab[2 * (n3 + 2) + k] = (invdXi * INV[k]) * (1.0 / 12.0);
        tab[3 * (n3 + 2) + k] = (Re * dXi) * JAC[k];
    }
    e = cudaMemcpyAsync(c->tabs, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    std::vector<float> tabf(tab.begin(), tab.end());
    if (e == cudaSuccess && c->mixed)
        e = cudaMemcpyAsync(c->tabf, tabf.data(), tabf.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { fail(nullptr, "table upload", e); chan_free(c); return CHAN_ECUDA; }

    chan::KParams &k = c->kp;
    k.n1 = n1; k.n2 = n2; k.n3 = n3; k.px = c->px; k.NJ = c->NJ;
    k.plane = c->plane; k.vol = c->vol;
    k.wp = c->wp; k.cs = c->cs;
    k.czh = c->tabs; k.cz8 = c->tabs + (n3 + 2); k.cz12 = c->tabs + 2 * (n3 + 2); k.pez = c->tabs + 3 * (n3 + 2);
    k.stat = c->stat; k.status = c->status; k.tacc = c->tacc; k.acc_on = 0; k.hwt = c->hwt;
    k.invRe = 1.0 / Re;
    k.ggM = gama * (gama - 1) * (Mac * Mac);
    k.ggMh = k.ggM * 0.5;
    k.gM2 = gama * (Mac * Mac);
    k.inv_gM2 = 1.0 / k.gM2;
    k.kq = gama * k.invRe * (1.0 / p->Pr);
    k.two3rd = 2.0 / 3.0;
    k.invdx = invdx; k.invdy = invdy;
    k.hdx = 0.5 * invdx; k.hdy = 0.5 * invdy;
    k.sx8 = invdx / 8.0; k.sx12 = invdx * (1.0 / 12.0);
    k.sy8 = invdy / 8.0; k.sy12 = invdy * (1.0 / 12.0);
    k.pex = Re * dx; k.pey = Re * dy;
    k.PexVal = p->Pe[0]; k.PeyVal = p->Pe[1]; k.pez_val = p->Pe[2];
    k.inv_dz1 = 1.0 / co[12]; k.inv_dzN = 1.0 / co[13];
    k.tabf = c->tabf;
    k.cd = chan::FluxC<double>{k.invRe, k.ggM, k.two3rd, k.kq, k.inv_gM2, k.hdx, k.hdy, k.sx8, k.sx12, k.sy8,
                               k.sy12, k.pex, k.pey, k.PexVal, k.PeyVal, k.pez_val};
    k.cf = chan::FluxC<float>{(float)k.invRe, (float)k.ggM, (float)k.two3rd, (float)k.kq, (float)k.inv_gM2,
                              (float)k.hdx, (float)k.hdy, (float)k.sx8, (float)k.sx12, (float)k.sy8,
                              (float)k.sy12, (float)k.pex, (float)k.pey, (float)k.PexVal, (float)k.PeyVal,
                              (float)k.pez_val};
    k.Twb = p->Tw[0]; k.Twt = p->Tw[1];
    k.muwb = pow(p->Tw[0], 0.7); k.muwt = pow(p->Tw[1], 0.7);
    for (int m = 0; m < 3; m++) {
        k.f1[m] = co[m]; k.f2[m] = co[3 + m]; k.b1[m] = co[6 + m]; k.b2[m] = co[9 + m];
    }
    k.force_on = p->forcing == CHAN_FORCE_WALLSHEAR ? 1 : 0;
    k.wall_custom = 0;
    k.ri = 0.0; k.tref = 1.0; k.buoy_on = 0;
    k.clk = nullptr;
    for (int w = 0; w < 2; w++) {
        k.wbc[w] = chan::WallBC{};
        k.wbc[w].Tw = p->Tw[w];
    }

    // stage-kernel launch shape: the default tile, k-chunks filling whole waves
    for (const StageSet &ss : kStageSets)
        for (int b = 0; b < 2 && e == cudaSuccess; b++)
            for (int v = 0; v < 4 && e == cudaSuccess; v++)
                e = cudaFuncSetAttribute((const void *)ss.k[b][v], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(v == 0 ? ss.smem : ss.smemf));
    if (e != cudaSuccess) { fail(nullptr, "cudaFuncSetAttribute", e); chan_free(c); return CHAN_ECUDA; }
    memset(c->tmd, 0, sizeof(c->tmd));
    memset(c->tmf, 0, sizeof(c->tmf));
    memset(c->tmb, 0, sizeof(c->tmb));
    for (int t = 0; t < CHAN_NTILES; t++) {
        const int ti = kStageSets[t].ti, tj = kStageSets[t].tj;
        for (int b = 0; b < 3 && !c->mixed; b++)
            if ((r = make_state_map(c, &c->tmd[t][b], c->q[b], false, ti, tj))) { g_init_error = c->err; chan_free(c); return r; }
        for (int b = 0; b < 2 && c->mixed; b++)
            if ((r = make_state_map(c, &c->tmf[t][b], c->qf[b], true, ti, tj))) { g_init_error = c->err; chan_free(c); return r; }
        // the tile's own points (no halo); the x origin 2 + TI*bx gives 16-byte aligned copies
        if ((r = make_state_map(c, &c->tmb[t], c->q[0], false, ti, tj, 0))) { g_init_error = c->err; chan_free(c); return r; }
    }
    if (set_launch(c, CHAN_TILE_32x8, 0) != CHAN_OK) { g_init_error = c->err; chan_free(c); return CHAN_ECUDA; }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    c->nsplit = stats_split(sms, n1, n2, n3);
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { fail(nullptr, "init sync", e); chan_free(c); return CHAN_ECUDA; }
    *out = c;
    return CHAN_OK;
}

int chan_upload(chan_ctx *c, const double *var, int64_t nstep, double time)
{
    if (!c || !var) return CHAN_EINVAL;
    CK(c, cudaSetDevice(c->dev));
    const size_t N = (size_t)c->n1 * c->n2 * c->n3, pl = (size_t)c->n1 * c->n2;
    // rho, u, v, w, E everywhere; T and p only where they are read: the two
    // wall planes and the four corner columns (the interior primitives are
    // derived from the conservative state)
    CK(c, cudaMemcpyAsync(c->dvar, var, 5 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    for (int m = 5; m < 7; m++) {
        for (size_t k : {(size_t)0, (size_t)c->n3 - 1})
            CK(c, cudaMemcpyAsync(c->dvar + m * N + k * pl, var + m * N + k * pl, pl * sizeof(double),
                                  cudaMemcpyHostToDevice, c->stream));
        for (size_t jc : {(size_t)0, (size_t)c->n2 - 1})
            for (size_t ic : {(size_t)0, (size_t)c->n1 - 1}) {
                const size_t o = m * N + jc * c->n1 + ic;
                CK(c, cudaMemcpy2DAsync(c->dvar + o, pl * sizeof(double), var + o, pl * sizeof(double),
                                        sizeof(double), c->n3, cudaMemcpyHostToDevice, c->stream));
            }
    }
    chan::k_upload<<<1184, 256, 0, c->stream>>>(c->kp, c->dvar, c->q[0], c->mixed ? c->q[0] : c->q[1],
                                                  c->mixed ? nullptr : c->q[2], c->cs);
    CK(c, cudaGetLastError());
    {
        dim3 block(32, 8), grid((c->n1 + 2 + 31) / 32, (c->n2 + 2 + 7) / 8, c->n3 - 2);
        chan::k_fill_ghosts<<<grid, block, 0, c->stream>>>(c->kp, c->q[0]);
        CK(c, cudaGetLastError());
        dim3 g2((c->n1 + 2 + 31) / 32, (c->n2 + 2 + 7) / 8, 2);
        chan::k_fill_wall_ring<<<g2, block, 0, c->stream>>>(c->kp);
        CK(c, cudaGetLastError());
    }
    { int r = seed_float_stages(c); if (r) return r; }
    CK(c, cudaMemsetAsync(c->stat, 0, (23 * (size_t)c->n3 + 2) * sizeof(double), c->stream));
    CK(c, cudaMemsetAsync(c->status, 0, sizeof(chan::DevStatus), c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    c->nstep = nstep;
    c->time = time;
    c->sync_nstep = nstep;
    c->sync_time = time;
    c->cur = 0;
    c->uploaded = true;
    c->sgs_valid = false;
    return CHAN_OK;
}

int chan_stage(chan_ctx *c, int iter)
{
    if (!c) return CHAN_EINVAL;
    if (!c->uploaded) { c->err = "chan_stage before chan_upload"; return CHAN_ESTATE; }
    if (iter < 1 || iter > c->nstage) { c->err = "iter out of range"; return CHAN_EINVAL; }
    if (c->mixed) { c->err = "the mixed-precision path runs whole steps only (chan_step)"; return CHAN_ESTATE; }
    CK(c, cudaSetDevice(c->dev));
    int r = launch_stage(c, iter, iter == c->nstage, c->nstep + 1, c->time + c->p.dt);
    if (r) return r;
    return read_status(c, nullptr);
}

int chan_step_async(chan_ctx *c, int nsteps)
{
    if (!c || nsteps < 0) return CHAN_EINVAL;
    if (!c->uploaded) { c->err = "chan_step before chan_upload"; return CHAN_ESTATE; }
    CK(c, cudaSetDevice(c->dev));
    return enqueue_steps(c, nsteps);
}

int chan_step(chan_ctx *c, int nsteps)
{
    int r = chan_step_async(c, nsteps);
    if (r) return r;
    return read_status(c, nullptr);
}

int chan_check(chan_ctx *c)
{
    if (!c) return CHAN_EINVAL;
    if (!c->uploaded) return CHAN_ESTATE;
    CK(c, cudaSetDevice(c->dev));
    c->kp.step = c->nstep;
    chan::k_check<<<1184, 256, 0, c->stream>>>(c->kp, c->q[c->cur]);
    CK(c, cudaGetLastError());
    return read_status(c, nullptr);
}

int chan_tau_wall(chan_ctx *c)
{
    if (!c) return CHAN_EINVAL;
    if (!c->uploaded) return CHAN_ESTATE;
    CK(c, cudaSetDevice(c->dev));
    int r = launch_stats(c, c->nstep, 0, 1);
    if (r) return r;
    CK(c, cudaStreamSynchronize(c->stream));
    return CHAN_OK;
}

int chan_avg_spatial(chan_ctx *c)
{
    if (!c) return CHAN_EINVAL;
    if (!c->uploaded) return CHAN_ESTATE;
    CK(c, cudaSetDevice(c->dev));
    int r = launch_stats(c, c->nstep, 1, 0);
    if (r) return r;
    CK(c, cudaStreamSynchronize(c->stream));
    return CHAN_OK;
}

int chan_stats(chan_ctx *c, double *tau2, double *stat1, double *stat2, double *corr)
{
    if (!c) return CHAN_EINVAL;
    CK(c, cudaSetDevice(c->dev));
    const size_t n3 = (size_t)c->n3;
    if (tau2) CK(c, cudaMemcpyAsync(tau2, c->stat + 23 * n3, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (stat1) CK(c, cudaMemcpyAsync(stat1, c->stat, 7 * n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (stat2) CK(c, cudaMemcpyAsync(stat2, c->stat + 7 * n3, 7 * n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (corr) CK(c, cudaMemcpyAsync(corr, c->stat + 14 * n3, 9 * n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return CHAN_OK;
}

int chan_set_forcing(chan_ctx *c, double tauL, double tauU, const double *rhobar)
{
    if (!c || !rhobar) return CHAN_EINVAL;
    CK(c, cudaSetDevice(c->dev));
    const size_t n3 = (size_t)c->n3;
    double tau[2] = {tauL, tauU};
    CK(c, cudaMemcpyAsync(c->stat + 23 * n3, tau, 2 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaMemcpyAsync(c->stat, rhobar, n3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return CHAN_OK;
}

int chan_download(chan_ctx *c, double *var)
{
    if (!c || !var) return CHAN_EINVAL;
    if (!c->uploaded) return CHAN_ESTATE;
    CK(c, cudaSetDevice(c->dev));
    const size_t N = (size_t)c->n1 * c->n2 * c->n3;
    chan::k_download<<<1184, 256, 0, c->stream>>>(c->kp, c->q[c->cur], c->dvar);
    CK(c, cudaGetLastError());
    CK(c, cudaMemcpyAsync(var, c->dvar, 7 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return CHAN_OK;
}

int chan_status(chan_ctx *c, int32_t *ijk, int64_t *nstep, double *time)
{
    if (!c) return CHAN_EINVAL;
    CK(c, cudaSetDevice(c->dev));
    int r = read_status(c, ijk);
    if (nstep) *nstep = c->nstep;
    if (time) *time = c->time;
    return r;
}

int chan_sync(chan_ctx *c)
{
    if (!c) return CHAN_EINVAL;
    CK(c, cudaSetDevice(c->dev));
    return read_status(c, nullptr);
}

int chan_profile(chan_ctx *c, int enable)
{
    if (!c) return CHAN_EINVAL;
    CK(c, cudaStreamSynchronize(c->stream));
    for (auto &pp : c->prof_pairs) { c->ev_pool.push_back(pp.a); c->ev_pool.push_back(pp.b); }
    c->prof_pairs.clear();
    c->prof = enable != 0;
    return CHAN_OK;
}

int chan_profile_read(chan_ctx *c, double *ms3, int64_t *count3)
{
    if (!c) return CHAN_EINVAL;
    CK(c, cudaStreamSynchronize(c->stream));
    double ms[3] = {0, 0, 0};
    int64_t cnt[3] = {0, 0, 0};
    for (auto &pp : c->prof_pairs) {
        float t = 0.f;
        CK(c, cudaEventElapsedTime(&t, pp.a, pp.b));
        ms[pp.cls] += t;
        cnt[pp.cls] += 1;
    }
    for (int m = 0; m < 3; m++) {
        if (ms3) ms3[m] = ms[m];
        if (count3) count3[m] = cnt[m];
    }
    return CHAN_OK;
}

void *chan_stream(chan_ctx *c) { return c ? (void *)c->stream : nullptr; }

int chan_selftest_pow07(const double *T, double *mine, double *libm, int64_t n, int32_t device)
{
    if (!T || !mine || !libm || n <= 0) return CHAN_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return CHAN_ECUDA;
    double *d = nullptr;
    const size_t b = (size_t)n * sizeof(double);
    if (cudaMalloc((void **)&d, 3 * b) != cudaSuccess) return CHAN_ENOMEM;
    cudaError_t e = cudaMemcpy(d, T, b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        chan::k_selftest_pow07<<<256, 256>>>(d, d + n, d + 2 * n, (long long)n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(mine, d + n, b, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(libm, d + 2 * n, b, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) { g_init_error = cudaGetErrorString(e); return CHAN_ECUDA; }
    return CHAN_OK;
}

int64_t chan_device_bytes(chan_ctx *c) { return c ? (int64_t)c->dev_bytes : 0; }

// ---------------------------------------------------------------------------
// Exact checkpoint of the device state: the conservative state with its
// ghosts, the wall planes, the stale corner columns, the forcing/statistics
// state and the counters, in native byte order.
namespace {
const char kCkpMagic[8] = {'C', 'H', 'A', 'N', 'C', 'K', 'P', '2'};
struct CkpHeader {
    char magic[8];
    int32_t nP[3];
    int32_t px;
    int64_t nstep;
    double time;
    int64_t tavg_samples;
    double tavg_t0, tavg_t1;
    int32_t acc_on;
    int32_t pad;
    // the run's physics and method: a restart into a context that differs in
    // any of them is refused instead of continuing with other physics
    double Re, Mac, dt, Pr, gama, Pe[3], Lx, Ly, Tw[2];
    int32_t rk_scheme, forcing, flags, pad2;
    uint64_t x3_hash;   // FNV-1a of the x3 mesh bytes given to chan_init
};

uint64_t fnv1a(const void *data, size_t n)
{
    const unsigned char *b = static_cast<const unsigned char *>(data);
    uint64_t h = 1469598103934665603ULL;
    for (size_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= 1099511628211ULL;
    }
    return h;
}

void ckp_fill_physics(const chan_ctx *c, CkpHeader &h)
{
    const chan_params &p = c->p;
    h.Re = p.Re; h.Mac = p.Mac; h.dt = p.dt; h.Pr = p.Pr; h.gama = p.gama;
    for (int m = 0; m < 3; m++) h.Pe[m] = p.Pe[m];
    h.Lx = p.Lx; h.Ly = p.Ly; h.Tw[0] = p.Tw[0]; h.Tw[1] = p.Tw[1];
    h.rk_scheme = p.rk_scheme; h.forcing = p.forcing; h.flags = p.flags;
    h.x3_hash = fnv1a(c->hx3.data(), c->hx3.size() * sizeof(double));
}

// name of the first physics field in which two headers differ, or nullptr
const char *ckp_physics_mismatch(const CkpHeader &a, const CkpHeader &b)
{
    if (a.Re != b.Re) return "Re";
    if (a.Mac != b.Mac) return "Mac";
    if (a.dt != b.dt) return "dt";
    if (a.Pr != b.Pr) return "Pr";
    if (a.gama != b.gama) return "gama";
    for (int m = 0; m < 3; m++)
        if (a.Pe[m] != b.Pe[m]) return "Pe";
    if (a.Lx != b.Lx || a.Ly != b.Ly) return "Lx/Ly";
    if (a.Tw[0] != b.Tw[0] || a.Tw[1] != b.Tw[1]) return "Tw";
    if (a.rk_scheme != b.rk_scheme) return "rk_scheme";
    if (a.forcing != b.forcing) return "forcing";
    if (a.flags != b.flags) return "flags (precision)";
    if (a.x3_hash != b.x3_hash) return "x3 mesh";
    return nullptr;
}
}  // namespace

int chan_checkpoint_write(chan_ctx *c, const char *path)
{
    if (!c || !path) return CHAN_EINVAL;
    if (!c->uploaded) { c->err = "checkpoint before chan_upload"; return CHAN_ESTATE; }
    if (c->cur != 0) { c->err = "checkpoint only between time steps"; return CHAN_ESTATE; }
    int r = read_status(c, nullptr);
    if (r == CHAN_BLOWUP) { c->err = "state blew up; no checkpoint"; return CHAN_ESTATE; }
    CK(c, cudaSetDevice(c->dev));
    CkpHeader h{};
    memcpy(h.magic, kCkpMagic, 8);
    for (int m = 0; m < 3; m++) h.nP[m] = c->p.nP[m];
    h.px = c->px; h.nstep = c->nstep; h.time = c->time;
    h.tavg_samples = c->tavg_samples; h.tavg_t0 = c->tavg_t0; h.tavg_t1 = c->tavg_t1; h.acc_on = c->kp.acc_on;
    ckp_fill_physics(c, h);
    const size_t nq = 5 * (size_t)c->vol, nw = 16 * (size_t)c->plane, ncs = (size_t)(c->n3 + 2) * 28,
                 nst = 23 * (size_t)c->n3 + 2;
    std::vector<double> hb(nq + nw + ncs + 2 * nst);
    double *o = hb.data();
    CK(c, cudaMemcpyAsync(o, c->q[0], nq * sizeof(double), cudaMemcpyDeviceToHost, c->stream)); o += nq;
    CK(c, cudaMemcpyAsync(o, c->wp, nw * sizeof(double), cudaMemcpyDeviceToHost, c->stream)); o += nw;
    CK(c, cudaMemcpyAsync(o, c->cs, ncs * sizeof(double), cudaMemcpyDeviceToHost, c->stream)); o += ncs;
    CK(c, cudaMemcpyAsync(o, c->stat, nst * sizeof(double), cudaMemcpyDeviceToHost, c->stream)); o += nst;
    CK(c, cudaMemcpyAsync(o, c->tacc, nst * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    FILE *f = fopen(path, "wb");
    if (!f) { c->err = std::string("cannot open ") + path; return CHAN_EIO; }
    bool ok = fwrite(&h, sizeof(h), 1, f) == 1 && fwrite(hb.data(), sizeof(double), hb.size(), f) == hb.size();
    ok = (fclose(f) == 0) && ok;
    if (!ok) { c->err = std::string("write failed: ") + path; return CHAN_EIO; }
    return CHAN_OK;
}

int chan_checkpoint_read(chan_ctx *c, const char *path)
{
    if (!c || !path) return CHAN_EINVAL;
    CK(c, cudaSetDevice(c->dev));
    FILE *f = fopen(path, "rb");
    if (!f) { c->err = std::string("cannot open ") + path; return CHAN_EIO; }
    CkpHeader h{};
    if (fread(&h, sizeof(h), 1, f) != 1 || memcmp(h.magic, kCkpMagic, 8) != 0) {
        fclose(f);
        c->err = std::string("not a checkpoint of this library: ") + path;
        return CHAN_EIO;
    }
    if (h.nP[0] != c->p.nP[0] || h.nP[1] != c->p.nP[1] || h.nP[2] != c->p.nP[2] || h.px != c->px) {
        fclose(f);
        c->err = "checkpoint grid differs from the context's";
        return CHAN_EINVAL;
    }
    {
        CkpHeader mine{};
        ckp_fill_physics(c, mine);
        if (const char *what = ckp_physics_mismatch(h, mine)) {
            fclose(f);
            c->err = std::string("checkpoint physics differ from the context's: ") + what;
            return CHAN_EINVAL;
        }
    }
    const size_t nq = 5 * (size_t)c->vol, nw = 16 * (size_t)c->plane, ncs = (size_t)(c->n3 + 2) * 28,
                 nst = 23 * (size_t)c->n3 + 2;
    std::vector<double> hb(nq + nw + ncs + 2 * nst);
    const bool ok = fread(hb.data(), sizeof(double), hb.size(), f) == hb.size();
    fclose(f);
    if (!ok) { c->err = std::string("checkpoint truncated: ") + path; return CHAN_EIO; }
    const double *o = hb.data();
    for (int b = 0; b < (c->mixed ? 1 : 3); b++)
        CK(c, cudaMemcpyAsync(c->q[b], o, nq * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    { int r = seed_float_stages(c); if (r) return r; }
    o += nq;
    CK(c, cudaMemcpyAsync(c->wp, o, nw * sizeof(double), cudaMemcpyHostToDevice, c->stream)); o += nw;
    CK(c, cudaMemcpyAsync(c->cs, o, ncs * sizeof(double), cudaMemcpyHostToDevice, c->stream)); o += ncs;
    CK(c, cudaMemcpyAsync(c->stat, o, nst * sizeof(double), cudaMemcpyHostToDevice, c->stream)); o += nst;
    CK(c, cudaMemcpyAsync(c->tacc, o, nst * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaMemsetAsync(c->status, 0, sizeof(chan::DevStatus), c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    c->nstep = h.nstep; c->time = h.time; c->sync_nstep = h.nstep; c->sync_time = h.time;
    c->tavg_samples = h.tavg_samples; c->tavg_t0 = h.tavg_t0; c->tavg_t1 = h.tavg_t1; c->kp.acc_on = h.acc_on;
    c->epoch++;
    c->cur = 0;
    c->uploaded = true;
    c->sgs_valid = false;
    return CHAN_OK;
}

int chan_set_buoyancy(chan_ctx *c, double Ri, double Tref)
{
    if (!c) return CHAN_EINVAL;
    if (!std::isfinite(Ri) || !std::isfinite(Tref)) { c->err = "Ri and Tref must be finite"; return CHAN_EINVAL; }
    c->kp.ri = Ri;
    c->kp.tref = Tref;
    c->kp.buoy_on = Ri != 0.0 ? 1 : 0;
    c->epoch++;
    return CHAN_OK;
}

int chan_set_closure(chan_ctx *c, chan_closure *m, int32_t on)
{
    if (!c) return CHAN_EINVAL;
    if (on < 0 || on > 2 || (on && !m)) return CHAN_EINVAL;
    if (on && c->mixed) { c->err = "the closure runs on plain FP64 contexts"; return CHAN_EINVAL; }
    CK(c, cudaSetDevice(c->dev));
    if (on && chan_internal_closure_device(m) != c->dev) { c->err = "closure on another device"; return CHAN_EINVAL; }
    if (on && !c->sgsX) {
        const long long n = (long long)(c->n1 - 2) * (c->n2 - 2) * (c->n3 - 2);
        int r = ensure_dx3(c);
        if (r) return r;
        CK(c, cudaMalloc((void **)&c->sgsX, (size_t)n * chan::kSgsIn * sizeof(float)));
        CK(c, cudaMalloc((void **)&c->sgsY, (size_t)n * chan::kSgsOut * sizeof(float)));
        CK(c, cudaMalloc((void **)&c->sgsS, (size_t)n * 4 * sizeof(double)));
        CK(c, cudaMalloc((void **)&c->sgsflag, sizeof(int)));
        CK(c, cudaMemset(c->sgsflag, 0, sizeof(int)));
        c->dev_bytes += (size_t)n * ((chan::kSgsIn + chan::kSgsOut) * sizeof(float) + 4 * sizeof(double)) + sizeof(int);
    }
    c->cl = on ? m : nullptr;
    c->closure_on = on != 0;
    c->closure_every_stage = on == 2;
    c->sgs_valid = false;
    c->epoch++;
    return CHAN_OK;
}

int chan_closure_flag(chan_ctx *c, int32_t *flag, int32_t reset)
{
    if (!c || !flag) return CHAN_EINVAL;
    *flag = 0;
    if (!c->sgsflag) return CHAN_OK;
    CK(c, cudaSetDevice(c->dev));
    CK(c, cudaMemcpyAsync(c->h_status, c->sgsflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    *flag = *(const int *)c->h_status;
    if (reset) CK(c, cudaMemsetAsync(c->sgsflag, 0, sizeof(int), c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return CHAN_OK;
}

int chan_set_launch(chan_ctx *c, int32_t tile, int32_t nchunks)
{
    if (!c) return CHAN_EINVAL;
    CK(c, cudaSetDevice(c->dev));
    return set_launch(c, tile, nchunks);
}

int chan_get_launch(chan_ctx *c, int32_t *tile, int32_t *nchunks, int32_t *kchunk)
{
    if (!c) return CHAN_EINVAL;
    if (tile) *tile = c->tile;
    if (nchunks) *nchunks = c->nchunks;
    if (kchunk) *kchunk = c->kchunk;
    return CHAN_OK;
}

int chan_set_wall_bc(chan_ctx *c, int32_t wall, const chan_wall_bc *bc)
{
    if (!c || !bc || wall < 0 || wall > 1) return CHAN_EINVAL;
    if (bc->velocity < CHAN_WALL_NOSLIP || bc->velocity > CHAN_WALL_WAVE ||
        (bc->thermal != CHAN_WALL_ISOTHERMAL && bc->thermal != CHAN_WALL_FIXED_GRADIENT)) {
        c->err = "bad wall-BC kind";
        return CHAN_EINVAL;
    }
    if ((bc->velocity == CHAN_WALL_SLIP_MASK && !bc->mask) || (bc->velocity == CHAN_WALL_UV_FIELD && !bc->uv)) {
        c->err = "wall-BC kind needs its mask / uv array";
        return CHAN_EINVAL;
    }
    if (bc->thermal == CHAN_WALL_ISOTHERMAL && !(bc->Tw > 0)) { c->err = "Tw must be > 0"; return CHAN_EINVAL; }
    CK(c, cudaSetDevice(c->dev));
    const size_t n12 = (size_t)c->n1 * c->n2;
    if (!c->wmask[wall]) {
        CK(c, cudaMalloc((void **)&c->wmask[wall], n12));
        CK(c, cudaMalloc((void **)&c->wuv[wall], 2 * n12 * sizeof(double)));
        CK(c, cudaMalloc((void **)&c->wx1[wall], (size_t)c->n1 * sizeof(double)));
        c->dev_bytes += n12 + 2 * n12 * sizeof(double) + (size_t)c->n1 * sizeof(double);
    }
    if (bc->mask) CK(c, cudaMemcpy(c->wmask[wall], bc->mask, n12, cudaMemcpyHostToDevice));
    if (bc->uv) CK(c, cudaMemcpy(c->wuv[wall], bc->uv, 2 * n12 * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<double> x1(c->n1);
    if (bc->x1) {
        for (int i = 0; i < c->n1; i++) x1[i] = bc->x1[i];
    } else {  // x1(1)=0, x1(i+1)=x1(i)+dx (v1.9/codes/comdata.f90:93-95)
        const double dx = c->p.Lx / (double)(c->n1 - 1);
        x1[0] = 0.0;
        for (int i = 1; i < c->n1; i++) x1[i] = x1[i - 1] + dx;
    }
    CK(c, cudaMemcpy(c->wx1[wall], x1.data(), x1.size() * sizeof(double), cudaMemcpyHostToDevice));
    chan::WallBC &W = c->kp.wbc[wall];
    W.vel = bc->velocity;
    W.therm = bc->thermal;
    W.Tw = bc->Tw;
    W.dTdz = bc->dTdz;
    W.g = bc->slip_grad;
    W.A = bc->wave[0]; W.kx = bc->wave[1]; W.om = bc->wave[2]; W.ph = bc->wave[3];
    W.mask = c->wmask[wall];
    W.uv = c->wuv[wall];
    W.x1 = c->wx1[wall];
    if (wall == 0) { c->kp.Twb = bc->Tw; c->kp.muwb = pow(bc->Tw, 0.7); }
    else { c->kp.Twt = bc->Tw; c->kp.muwt = pow(bc->Tw, 0.7); }
    c->kp.wall_custom = 0;
    for (int w = 0; w < 2; w++)
        if (c->kp.wbc[w].vel != 0 || c->kp.wbc[w].therm != 0) c->kp.wall_custom = 1;
    c->epoch++;
    return CHAN_OK;
}

int chan_time_avg_start(chan_ctx *c)
{
    if (!c) return CHAN_EINVAL;
    CK(c, cudaSetDevice(c->dev));
    CK(c, cudaMemsetAsync(c->tacc, 0, (23 * (size_t)c->n3 + 2) * sizeof(double), c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    c->tavg_samples = 0;
    c->kp.acc_on = 1;
    c->epoch++;
    return CHAN_OK;
}

int chan_time_avg(chan_ctx *c, double *sum1, double *sum2, double *sumc, double *sumtau, int64_t *nsamples,
                  double *t0, double *t1)
{
    if (!c) return CHAN_EINVAL;
    CK(c, cudaSetDevice(c->dev));
    const size_t n3 = (size_t)c->n3;
    if (sum1) CK(c, cudaMemcpyAsync(sum1, c->tacc, 7 * n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (sum2) CK(c, cudaMemcpyAsync(sum2, c->tacc + 7 * n3, 7 * n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (sumc) CK(c, cudaMemcpyAsync(sumc, c->tacc + 14 * n3, 9 * n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (sumtau) CK(c, cudaMemcpyAsync(sumtau, c->tacc + 23 * n3, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    if (nsamples) *nsamples = c->tavg_samples;
    if (t0) *t0 = c->tavg_t0;
    if (t1) *t1 = c->tavg_t1;
    return CHAN_OK;
}

int chan_avg_spatial_noalloc(const double *var, const int32_t *nP, double *stat1, double *stat2, double *corr,
                             int32_t device)
{
    g_init_error.clear();
    if (!var || !nP || !stat1 || !stat2 || !corr) { g_init_error = "NULL argument"; return CHAN_EINVAL; }
    const int n1 = nP[0], n2 = nP[1], n3 = nP[2];
    if (n1 < 1 || n2 < 1 || n3 < 1) { g_init_error = "every nP must be >= 1"; return CHAN_EINVAL; }
    const long long pl = (long long)n1 * n2;
    const long long head = (23LL * n3 + 31) / 32 * 32;
    if (head + 7 * pl > (long long)CHAN_NOALLOC_MAX_DOUBLES) {
        char buf[256];
        snprintf(buf, sizeof(buf),
                 "chan_avg_spatial_noalloc: 23*nP3 + 7*nP1*nP2 = %lld doubles exceeds the fixed area of %d doubles",
                 head + 7 * pl, (int)CHAN_NOALLOC_MAX_DOUBLES);
        g_init_error = buf;
        return CHAN_EINVAL;
    }
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { g_init_error = std::string("cudaSetDevice: ") + cudaGetErrorString(e); return CHAN_ECUDA; }
    double *scr = noalloc_scratch();
    if (!scr) { cudaSetDevice(prev); return CHAN_ECUDA; }
    double *res = scr, *slab = scr + head;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int S = stats_split(sms, n1, n2, n3);
    const long long kslab_ll = ((long long)CHAN_NOALLOC_MAX_DOUBLES - head) / (7 * pl);
    const int kslab = (int)(kslab_ll < n3 ? kslab_ll : n3);
    // the results must start at zero: every plane is written below, and a
    // failed call must not hand back the previous call's numbers
    e = cudaMemsetAsync(res, 0, 23 * (size_t)n3 * sizeof(double), 0);
    for (int k0 = 0; k0 < n3 && e == cudaSuccess; k0 += kslab) {
        const int nk = (n3 - k0) < kslab ? (n3 - k0) : kslab;
        for (int m = 0; m < 7 && e == cudaSuccess; m++)
            e = cudaMemcpyAsync(slab + (size_t)m * nk * pl, var + ((size_t)m * n3 + k0) * pl,
                                (size_t)nk * pl * sizeof(double), cudaMemcpyHostToDevice, 0);
        if (e == cudaSuccess) {
            k_moments_slab<<<nk, chan::kStatThreads, 0, 0>>>(slab, n1, n2, nk, k0, n3, S, res);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(stat1, res, 7 * (size_t)n3 * sizeof(double), cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(stat2, res + 7 * (size_t)n3, 7 * (size_t)n3 * sizeof(double), cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(corr, res + 14 * (size_t)n3, 9 * (size_t)n3 * sizeof(double), cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    cudaSetDevice(prev);
    if (e != cudaSuccess) { g_init_error = std::string("chan_avg_spatial_noalloc: ") + cudaGetErrorString(e); return CHAN_ECUDA; }
    return CHAN_OK;
}

int chan_diag_enable(chan_ctx *c, const int32_t *planes, int32_t nplanes, int32_t every, const double *x3q,
                     double x2end, int32_t capacity)
{
    if (!c) return CHAN_EINVAL;
    if (every < 0 || nplanes < 0 || nplanes > CHAN_DIAG_MAX_PLANES || (nplanes > 0 && !planes) || capacity < 0) {
        c->err = "chan_diag_enable: bad arguments";
        return CHAN_EINVAL;
    }
    CK(c, cudaSetDevice(c->dev));
    CK(c, cudaStreamSynchronize(c->stream));
    if (every == 0) { c->diag_every = 0; c->diag_count = 0; return CHAN_OK; }
    if (capacity < 1) { c->err = "chan_diag_enable: capacity must be >= 1"; return CHAN_EINVAL; }
    if (!(x2end > 0)) { c->err = "chan_diag_enable: x2end must be > 0"; return CHAN_EINVAL; }
    const int n3 = c->n3;
    const double *z = x3q ? x3q : c->hx3.data();
    if (!(z[n3 - 1] > 0)) { c->err = "chan_diag_enable: x3(nP3) must be > 0"; return CHAN_EINVAL; }
    if (c->diag_rec) { cudaFree(c->diag_rec); c->diag_rec = nullptr; }
    if (!c->diag_part) {
        CK(c, cudaMalloc((void **)&c->diag_part, (size_t)n3 * sizeof(double)));
        CK(c, cudaMalloc((void **)&c->diag_x3, (size_t)n3 * sizeof(double)));
        c->dev_bytes += 2 * (size_t)n3 * sizeof(double);
    }
    const int reclen = 3 + 3 * nplanes;
    CK(c, cudaMalloc((void **)&c->diag_rec, (size_t)capacity * reclen * sizeof(double)));
    CK(c, cudaMemcpy(c->diag_x3, z, (size_t)n3 * sizeof(double), cudaMemcpyHostToDevice));
    chan::DiagParams &D = c->dp;
    D.nplanes = nplanes;
    for (int m = 0; m < chan::kDiagMaxPlanes; m++) D.planes[m] = m < nplanes ? planes[m] : 0;
    D.x3q = c->diag_x3;
    D.dy = c->p.Ly / (double)(c->n2 - 1);
    D.Ayz = z[n3 - 1] * x2end;
    D.part = c->diag_part;
    c->diag_every = every;
    c->diag_cap = capacity;
    c->diag_reclen = reclen;
    c->diag_count = 0;
    return CHAN_OK;
}

int chan_diag_read(chan_ctx *c, double *records, int32_t max_records, int32_t *nrecords, int64_t *lost)
{
    if (!c || !nrecords) return CHAN_EINVAL;
    if (!c->diag_rec) { *nrecords = 0; if (lost) *lost = 0; return CHAN_OK; }
    CK(c, cudaSetDevice(c->dev));
    const long long avail = c->diag_count < c->diag_cap ? c->diag_count : c->diag_cap;
    if (!records) { *nrecords = (int32_t)avail; if (lost) *lost = c->diag_count - avail; return CHAN_OK; }
    if (max_records < avail) { c->err = "chan_diag_read: records buffer too small"; return CHAN_EINVAL; }
    std::vector<double> ring((size_t)c->diag_cap * c->diag_reclen);
    CK(c, cudaMemcpyAsync(ring.data(), c->diag_rec, ring.size() * sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    const long long first = c->diag_count - avail;  // index of the oldest record kept
    int32_t n = 0;
    for (long long r = first; r < c->diag_count; r++) {
        const double *src = ring.data() + (size_t)(r % c->diag_cap) * c->diag_reclen;
        if (src[0] < 0) continue;  // after a blow-up
        memcpy(records + (size_t)n * c->diag_reclen, src, c->diag_reclen * sizeof(double));
        n++;
    }
    *nrecords = n;
    if (lost) *lost = first;
    c->diag_count = 0;
    return CHAN_OK;
}

namespace {
int upload_coords(chan_ctx *c, const double *x1, const double *x2, const double *x3, double *dst)
{
    const int n1 = c->n1, n2 = c->n2, n3 = c->n3;
    std::vector<double> h((size_t)n1 + n2 + n3);
    for (int i = 0; i < n1; i++) h[i] = x1 ? x1[i] : 0.0;
    if (!x1) {  // x1(1)=0, x1(i+1)=x1(i)+dx (v1.9/codes/comdata.f90:93-95)
        const double dx = c->p.Lx / (double)(n1 - 1);
        for (int i = 1; i < n1; i++) h[i] = h[i - 1] + dx;
    }
    for (int j = 0; j < n2; j++) h[n1 + j] = x2 ? x2[j] : 0.0;
    if (!x2) {
        const double dy = c->p.Ly / (double)(n2 - 1);
        for (int j = 1; j < n2; j++) h[n1 + j] = h[n1 + j - 1] + dy;
    }
    for (int k = 0; k < n3; k++) h[n1 + n2 + k] = x3 ? x3[k] : c->hx3[k];
    CK(c, cudaMemcpyAsync(dst, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return CHAN_OK;
}
}  // namespace

int chan_fluctuation_q(chan_ctx *c, const double *mean, const double *x1, const double *x2, const double *x3,
                       double *fluc, double *qcrit)
{
    if (!c || !mean) return CHAN_EINVAL;
    if (!c->uploaded) return CHAN_ESTATE;
    CK(c, cudaSetDevice(c->dev));
    const size_t N = (size_t)c->n1 * c->n2 * c->n3;
    if (!c->dq) {
        CK(c, cudaMalloc((void **)&c->dq, (N + 7 * (size_t)c->n3) * sizeof(double)));
        CK(c, cudaMalloc((void **)&c->dxyz, ((size_t)c->n1 + c->n2 + c->n3) * sizeof(double)));
        c->dev_bytes += (N + 7 * (size_t)c->n3 + c->n1 + c->n2 + c->n3) * sizeof(double);
    }
    double *dmean = c->dq + N;
    int r = upload_coords(c, x1, x2, x3, c->dxyz);
    if (r) return r;
    CK(c, cudaMemcpyAsync(dmean, mean, 7 * (size_t)c->n3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    chan::k_download<<<1184, 256, 0, c->stream>>>(c->kp, c->q[c->cur], c->dvar);
    CK(c, cudaGetLastError());
    chan::k_fluctuation<<<1184, 256, 0, c->stream>>>(c->dvar, dmean, c->n1, c->n2, c->n3);
    CK(c, cudaGetLastError());
    if (qcrit) {
        chan::k_qcrit<<<1184, 256, 0, c->stream>>>(c->n1, c->n2, c->n3, c->dvar + N, c->dvar + 2 * N,
                                                    c->dvar + 3 * N, c->dxyz, c->dxyz + c->n1,
                                                    c->dxyz + c->n1 + c->n2, c->dq);
        CK(c, cudaGetLastError());
        CK(c, cudaMemcpyAsync(qcrit, c->dq, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    if (fluc) CK(c, cudaMemcpyAsync(fluc, c->dvar, 7 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return CHAN_OK;
}

int chan_q_criterion(const int32_t *nP, const double *u, const double *v, const double *w, const double *x1,
                     const double *x2, const double *x3, double *qcrit, int32_t device)
{
    g_init_error.clear();
    if (!nP || !u || !v || !w || !x1 || !x2 || !x3 || !qcrit) { g_init_error = "NULL argument"; return CHAN_EINVAL; }
    const long long n1 = nP[0], n2 = nP[1], n3 = nP[2];
    if (n1 < 1 || n2 < 1 || n3 < 1 || n1 * n2 * n3 > (1LL << 31)) { g_init_error = "bad nP"; return CHAN_EINVAL; }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { fail(nullptr, "cudaSetDevice", e); return CHAN_ECUDA; }
    const size_t N = (size_t)(n1 * n2 * n3);
    const size_t nc = (size_t)(n1 + n2 + n3);
    double *d = nullptr;
    int rc = CHAN_OK;
    e = cudaMalloc((void **)&d, (4 * N + nc) * sizeof(double));
    if (e != cudaSuccess) { fail(nullptr, "cudaMalloc", e); cudaSetDevice(prev); return CHAN_ENOMEM; }
    cudaStream_t st = nullptr;
    e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, u, N * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d + N, v, N * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d + 2 * N, w, N * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d + 4 * N, x1, n1 * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d + 4 * N + n1, x2, n2 * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d + 4 * N + n1 + n2, x3, n3 * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        chan::k_qcrit<<<1184, 256, 0, st>>>((int)n1, (int)n2, (int)n3, d, d + N, d + 2 * N, d + 4 * N,
                                            d + 4 * N + n1, d + 4 * N + n1 + n2, d + 3 * N);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(qcrit, d + 3 * N, N * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = fail(nullptr, "chan_q_criterion", e);
    if (st) cudaStreamDestroy(st);
    cudaFree(d);
    cudaSetDevice(prev);
    return rc;
}

int chan_debug_canaries(chan_ctx *c, int64_t *corrupted)
{
    if (!c || !corrupted) return CHAN_EINVAL;
    CK(c, cudaSetDevice(c->dev));
    CK(c, cudaStreamSynchronize(c->stream));
    int64_t bad = 0;
    std::vector<unsigned long long> h(kGuard);
    for (const auto &g : c->guarded) {
        for (int side = 0; side < 2; side++) {
            const double *src = side == 0 ? g.base : g.base + kGuard + g.n;
            CK(c, cudaMemcpy(h.data(), src, kGuard * sizeof(double), cudaMemcpyDeviceToHost));
            for (size_t w = 0; w < kGuard; w++) bad += h[w] != kCanary;
        }
    }
    *corrupted = bad;
    return CHAN_OK;
}

void chan_free(chan_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->dev);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto &pp : c->prof_pairs) { cudaEventDestroy(pp.a); cudaEventDestroy(pp.b); }
    for (auto e : c->ev_pool) cudaEventDestroy(e);
    for (auto &g : c->guarded) cudaFree(g.base);
    for (int w = 0; w < 2; w++) {
        if (c->wmask[w]) cudaFree(c->wmask[w]);
        if (c->wuv[w]) cudaFree(c->wuv[w]);
        if (c->wx1[w]) cudaFree(c->wx1[w]);
    }

    if (c->diag_rec) cudaFree(c->diag_rec);
    if (c->diag_part) cudaFree(c->diag_part);
    if (c->diag_x3) cudaFree(c->diag_x3);
    if (c->dq) cudaFree(c->dq);
    if (c->dx3) cudaFree(c->dx3);
    if (c->sgsX) cudaFree(c->sgsX);
    if (c->sgsY) cudaFree(c->sgsY);
    if (c->sgsS) cudaFree(c->sgsS);
    if (c->sgsflag) cudaFree(c->sgsflag);
    if (c->dxyz) cudaFree(c->dxyz);
    if (c->status) cudaFree(c->status);
    if (c->h_status) cudaFreeHost(c->h_status);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Ensembles: several contexts on one device stepped together.  Each member
// keeps its own stream, buffers, parameters and launch shape.  A block of L
// steps of every member (L = the least common multiple of their statistics
// cadences, so that each replay starts at the same phase of every cadence) is
// captured once into a CUDA graph with one branch per member; the graph is
// replayed for as many whole blocks as a call asks for, and the members'
// branches run concurrently, filling the GPU with small grids that alone
// would not.  Kernels replayed from the graph read the step number and time
// from a device clock per member (k_clock_advance moves it), since a graph's
// kernel arguments are fixed at capture.  Results are bit for bit those of
// stepping each member alone.

struct chan_ensemble {
    std::vector<chan_ctx *> m;
    int dev = 0;
    cudaStream_t origin = nullptr;
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> join;
    chan::DevClock *dclk = nullptr;   // [n] device clocks
    chan::DevClock *hclk = nullptr;   // [n] pinned staging for the clock upload
    cudaGraphExec_t exec = nullptr;
    int L = 1;                        // steps per replay
    std::vector<long long> cap_epoch, cap_phase;
    long long replays = 0, captures = 0;
    double last_ms = 0.0;             // device time of the last call's graph replays (CUDA events)
    std::string err;
    // persistent mode: one persistent kernel per block of L steps (k_ensemble)
    int mode = CHAN_ENSEMBLE_GRAPH;        // requested mode
    bool persistent = false;               // the captured graph holds the persistent kernel
    std::string fallback;                  // why the requested persistent mode fell back
    chan::PPhase *dph = nullptr;
    chan::PItem *ditems = nullptr;
    chan::KParams *dkps = nullptr;
    CUtensorMap *dmaps = nullptr;
    unsigned long long *dcnt = nullptr;    // [n] completed units per member, then the work-list position
    int *derr = nullptr, *herr = nullptr;
    size_t cap_ph = 0, cap_items = 0, cap_kps = 0, cap_maps = 0;
    long long nitems = 0;
    int pgrid = 0;
    bool stall_test = false;               // host-side fault injection for tests
};

namespace {

int efail(chan_ensemble *e, const char *what, cudaError_t r)
{
    e->err = std::string(what) + ": " + cudaGetErrorString(r);
    return CHAN_ECUDA;
}

#define EK(e, call)                                    \
    do {                                               \
        cudaError_t r_ = (call);                       \
        if (r_ != cudaSuccess) return efail((e), #call, r_); \
    } while (0)

long long gcd_ll(long long a, long long b)
{
    while (b) { const long long t = a % b; a = b; b = t; }
    return a;
}

long long member_phase(const chan_ctx *c) { return c->p.istat > 0 ? c->nstep % c->p.istat : 0; }

bool graph_valid(const chan_ensemble *e)
{
    if (!e->exec) return false;
    for (size_t i = 0; i < e->m.size(); i++)
        if (e->m[i]->epoch != e->cap_epoch[i] || member_phase(e->m[i]) != e->cap_phase[i]) return false;
    return true;
}

// origin waits for every member's queued work; members wait for the origin
int join_members_to_origin(chan_ensemble *e)
{
    for (size_t i = 0; i < e->m.size(); i++) {
        EK(e, cudaEventRecord(e->join[i], e->m[i]->stream));
        EK(e, cudaStreamWaitEvent(e->origin, e->join[i], 0));
    }
    return CHAN_OK;
}
int members_wait_origin(chan_ensemble *e)
{
    EK(e, cudaEventRecord(e->fork, e->origin));
    for (chan_ctx *c : e->m) EK(e, cudaStreamWaitEvent(c->stream, e->fork, 0));
    return CHAN_OK;
}

// (re)allocate a device array for n elements when it holds fewer
template <typename T>
cudaError_t ensure_dev(T **p, size_t *cap, size_t n)
{
    if (*p && *cap >= n) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    cudaError_t r = cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T));
    if (r == cudaSuccess) *cap = n;
    return r;
}

// why the members cannot run in the persistent kernel ("" if they can)
std::string persistent_blocker(const chan_ensemble *e)
{
    const bool mixed = e->m[0]->mixed;
    for (chan_ctx *c : e->m) {
        if (c->mixed != mixed) return "members of both precisions";
        if (c->closure_on) return "a member runs with the learned closure";
        if (c->tile != CHAN_TILE_32x8 && c->tile != CHAN_TILE_16x16) return "a member uses a tile of other than 256 threads";
    }
    long long recs = 0;
    for (chan_ctx *c : e->m) recs += c->nstage;
    if (recs > chan::kEnsKps) return "more parameter records than the persistent kernel's constant memory holds";
    return "";
}

// The work list of one block of L steps of every member for k_ensemble, its
// upload, and the graph of one block: reset the counters, one launch.
int build_persistent(chan_ensemble *e)
{
    const size_t n = e->m.size();
    const bool mixed = e->m[0]->mixed;
    std::vector<chan::KParams> kps;
    std::vector<CUtensorMap> maps, bmaps;   // per stage record: the input's map; per member: the RK base's
    std::vector<std::vector<chan::PPhase>> per(n);
    for (size_t i = 0; i < n; i++) {
        chan_ctx *c = e->m[i];
        const int kp0 = (int)kps.size();
        for (int it = 1; it <= c->nstage; it++) {
            set_stage(c, it);
            chan::KParams k = c->kp;
            k.check = it == c->nstage ? 1 : 0;
            k.clk = e->dclk + i;
            kps.push_back(k);
            maps.push_back(stage_map(c));
        }
        bmaps.push_back(c->tmb[c->tile]);
        unsigned long long need = 0;
        auto add = [&](chan::PPhase ph) {
            ph.member = (int)i;
            ph.need = need;
            need += (unsigned long long)ph.units;
            per[i].push_back(ph);
        };
        for (int s = 0; s < e->L; s++) {
            chan::PPhase ck{};
            ck.kind = chan::kPClock; ck.units = 1; ck.kp = kp0; ck.dt = c->p.dt;
            add(ck);
            for (int it = 1; it <= c->nstage; it++) {
                const bool last = it == c->nstage;
                chan::PPhase st{};
                st.kind = chan::kPStage;
                st.variant = !c->mixed ? 0 : (it == 1 ? 1 : (last ? 3 : 2));
                st.tile = c->tile;
                st.nx = c->ntx; st.ny = c->nty;
                st.units = c->ntx * c->nty * c->nchunks;
                st.kp = kp0 + it - 1;
                st.tm = nullptr;   // set after upload (index kp0 + it - 1 of the maps)
                add(st);
                chan::PPhase w{};
                w.kind = chan::kPWall;
                w.variant = (c->mixed && !last) ? 1 : 0;
                w.nx = (c->n1 + 2 + chan::kWallBX - 1) / chan::kWallBX;
                w.ny = (c->n2 + 2 + chan::kWallBY - 1) / chan::kWallBY;
                w.group = 8;
                w.units = (w.nx * w.ny * 2 + w.group - 1) / w.group;
                w.kp = kp0 + it - 1;
                add(w);
            }
            if (c->p.istat > 0 && (c->nstep + s + 1) % c->p.istat == 0) {
                chan::PPhase a{};
                a.kind = chan::kPStatsPart; a.nx = c->nsplit; a.units = (c->n3 + 2) * c->nsplit;
                a.kp = kp0 + c->nstage - 1; a.q = c->q[0]; a.part = c->spart;
                add(a);
                chan::PPhase b = a;
                b.kind = chan::kPStatsFin; b.units = (c->n3 + 2 + 7) / 8;
                add(b);
            }
        }
    }
    // the phases in one array; the units interleaved member by member, phase by phase
    std::vector<chan::PPhase> ph;
    std::vector<chan::PItem> items;
    std::vector<size_t> first(n);
    size_t maxp = 0;
    for (size_t i = 0; i < n; i++) {
        first[i] = ph.size();
        ph.insert(ph.end(), per[i].begin(), per[i].end());
        maxp = std::max(maxp, per[i].size());
    }
    for (size_t q = 0; q < maxp; q++)
        for (size_t i = 0; i < n; i++)
            if (q < per[i].size())
                for (int u = 0; u < per[i][q].units; u++) items.push_back({(int)(first[i] + q), u});
    const size_t nmaps = maps.size();
    maps.insert(maps.end(), bmaps.begin(), bmaps.end());
    EK(e, ensure_dev(&e->dmaps, &e->cap_maps, maps.size()));
    for (auto &f : ph)
        if (f.kind == chan::kPStage) {
            f.tm = e->dmaps + f.kp;
            f.tmb = e->dmaps + nmaps + f.member;
        }
    if (e->stall_test && !ph.empty()) {
        // host-side fault injection: member 0's first stage waits for a unit count never reached
        for (size_t k = 0; k < per[0].size(); k++)
            if (ph[first[0] + k].kind == chan::kPStage) { ph[first[0] + k].need = ~0ULL; break; }
    }
    EK(e, ensure_dev(&e->dph, &e->cap_ph, ph.size()));
    EK(e, ensure_dev(&e->ditems, &e->cap_items, items.size()));
    EK(e, ensure_dev(&e->dkps, &e->cap_kps, kps.size()));
    if (!e->dcnt) EK(e, cudaMalloc((void **)&e->dcnt, (n + 1) * sizeof(unsigned long long)));
    if (!e->derr) EK(e, cudaMalloc((void **)&e->derr, sizeof(int)));
    if (!e->herr) EK(e, cudaMallocHost((void **)&e->herr, sizeof(int)));
    EK(e, cudaMemcpyAsync(e->dmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, e->origin));
    EK(e, cudaMemcpyAsync(e->dph, ph.data(), ph.size() * sizeof(chan::PPhase), cudaMemcpyHostToDevice, e->origin));
    EK(e, cudaMemcpyAsync(e->ditems, items.data(), items.size() * sizeof(chan::PItem), cudaMemcpyHostToDevice,
                          e->origin));
    EK(e, cudaMemcpyAsync(e->dkps, kps.data(), kps.size() * sizeof(chan::KParams), cudaMemcpyHostToDevice, e->origin));
    EK(e, cudaMemsetAsync(e->derr, 0, sizeof(int), e->origin));
    EK(e, cudaStreamSynchronize(e->origin));   // the host vectors are temporaries
    e->nitems = (long long)items.size();

    const void *fn = mixed ? (const void *)chan::k_ensemble<true> : (const void *)chan::k_ensemble<false>;
    const size_t smem = mixed ? chan::PersistShape<true>::bytes : chan::PersistShape<false>::bytes;
    EK(e, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0, sms = 148;
    EK(e, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, smem));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->dev);
    e->pgrid = std::max(1, occ) * sms;

    chan::PPlan plan{};
    plan.phases = e->dph; plan.items = e->ditems; plan.nitems = e->nitems;
    plan.done = e->dcnt; plan.next = e->dcnt + n; plan.err = e->derr; plan.clk = e->dclk;
#ifdef CHAN_PERSIST_GLOBAL_KPS
    plan.kps = e->dkps;
#endif
    void *ckps = nullptr;
    EK(e, cudaGetSymbolAddress(&ckps, chan::c_ens_kps));
    EK(e, cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeThreadLocal));
    cudaError_t r = cudaMemcpyAsync(ckps, e->dkps, kps.size() * sizeof(chan::KParams), cudaMemcpyDeviceToDevice,
                                    e->origin);
    if (r == cudaSuccess) r = cudaMemsetAsync(e->dcnt, 0, (n + 1) * sizeof(unsigned long long), e->origin);
    if (r == cudaSuccess) {
        if (mixed)
            chan::k_ensemble<true><<<e->pgrid, 256, smem, e->origin>>>(plan);
        else
            chan::k_ensemble<false><<<e->pgrid, 256, smem, e->origin>>>(plan);
        r = cudaGetLastError();
    }
    cudaGraph_t g = nullptr;
    const cudaError_t re = cudaStreamEndCapture(e->origin, &g);
    if (r != cudaSuccess) { if (g) cudaGraphDestroy(g); return efail(e, "persistent capture", r); }
    if (re != cudaSuccess) return efail(e, "cudaStreamEndCapture", re);
    const cudaError_t ri = cudaGraphInstantiate(&e->exec, g, 0);
    cudaGraphDestroy(g);
    if (ri != cudaSuccess) { e->exec = nullptr; return efail(e, "cudaGraphInstantiate", ri); }
    return CHAN_OK;
}

// capture L steps of every member into one graph (host counters restored)
int build_graph(chan_ensemble *e)
{
    if (e->exec) { cudaGraphExecDestroy(e->exec); e->exec = nullptr; }
    e->persistent = false;
    e->fallback.clear();
    if (e->mode == CHAN_ENSEMBLE_PERSISTENT) {
        e->fallback = persistent_blocker(e);
        if (e->fallback.empty()) {
            const int rc = build_persistent(e);
            if (rc) return rc;
            for (size_t i = 0; i < e->m.size(); i++) {
                e->cap_epoch[i] = e->m[i]->epoch;
                e->cap_phase[i] = member_phase(e->m[i]);
            }
            e->persistent = true;
            e->captures++;
            return CHAN_OK;
        }
    }
    EK(e, cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeThreadLocal));
    int rc = CHAN_OK;
    cudaError_t r = cudaEventRecord(e->fork, e->origin);
    for (size_t i = 0; i < e->m.size() && rc == CHAN_OK && r == cudaSuccess; i++) {
        chan_ctx *c = e->m[i];
        r = cudaStreamWaitEvent(c->stream, e->fork, 0);
        if (r != cudaSuccess) break;
        const long long ns = c->nstep, tn = c->tavg_samples;
        const double tm = c->time, ta = c->tavg_t0, tb = c->tavg_t1;
        const int cur = c->cur;
        const bool prof = c->prof;
        c->prof = false;
        c->kp.clk = c->dclk;
        rc = enqueue_steps(c, e->L, kCapture);
        if (rc != CHAN_OK) e->err = c->err;
        c->kp.clk = nullptr;
        c->prof = prof;
        c->nstep = ns; c->time = tm; c->tavg_samples = tn; c->tavg_t0 = ta; c->tavg_t1 = tb; c->cur = cur;
        if (rc == CHAN_OK) r = cudaEventRecord(e->join[i], c->stream);
        if (rc == CHAN_OK && r == cudaSuccess) r = cudaStreamWaitEvent(e->origin, e->join[i], 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t re = cudaStreamEndCapture(e->origin, &g);
    if (rc != CHAN_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (r != cudaSuccess) { if (g) cudaGraphDestroy(g); return efail(e, "capture", r); }
    if (re != cudaSuccess) return efail(e, "cudaStreamEndCapture", re);
    const cudaError_t ri = cudaGraphInstantiate(&e->exec, g, 0);
    cudaGraphDestroy(g);
    if (ri != cudaSuccess) { e->exec = nullptr; return efail(e, "cudaGraphInstantiate", ri); }
    for (size_t i = 0; i < e->m.size(); i++) {
        e->cap_epoch[i] = e->m[i]->epoch;
        e->cap_phase[i] = member_phase(e->m[i]);
    }
    e->captures++;
    return CHAN_OK;
}

// one timed trial of the autotuner: every stage but the last of every
// member, reps times, all members concurrently; the state is not modified
// (only the stage buffers and the wall ring, which the caller restores)
int tune_trial(chan_ensemble *e, int reps, float *ms)
{
    int rc = members_wait_origin(e);
    if (rc) return rc;
    EK(e, cudaEventRecord(e->t0, e->origin));
    rc = members_wait_origin(e);
    if (rc) return rc;
    for (chan_ctx *c : e->m) {
        const int ns = c->nstage > 1 ? c->nstage - 1 : 1;
        for (int r = 0; r < reps; r++)
            for (int it = 1; it <= ns; it++) {
                rc = launch_stage(c, it, false, c->nstep + 1, c->time + c->p.dt);
                if (rc) { e->err = c->err; return rc; }
            }
    }
    rc = join_members_to_origin(e);
    if (rc) return rc;
    EK(e, cudaEventRecord(e->t1, e->origin));
    EK(e, cudaEventSynchronize(e->t1));
    EK(e, cudaEventElapsedTime(ms, e->t0, e->t1));
    *ms /= (float)reps;
    return CHAN_OK;
}

}  // namespace

extern "C" {

int chan_ensemble_create(chan_ctx *const *members, int32_t n, chan_ensemble **out)
{
    if (!members || n < 1 || !out) return CHAN_EINVAL;
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        if (!members[i] || members[i]->dclk) return CHAN_EINVAL;   // null, or already in an ensemble
        for (int j = 0; j < i; j++)
            if (members[j] == members[i]) return CHAN_EINVAL;
        if (members[i]->dev != members[0]->dev) return CHAN_EINVAL;
    }
    long long L = 1;
    for (int i = 0; i < n; i++) {
        const long long is = members[i]->p.istat > 0 ? members[i]->p.istat : 1;
        L = L / gcd_ll(L, is) * is;
        if (L > 10000) return CHAN_EINVAL;   // statistics cadences too far apart for one graph block
    }
    chan_ensemble *e = new chan_ensemble;
    e->m.assign(members, members + n);
    e->dev = members[0]->dev;
    e->L = (int)L;
    e->join.assign(n, nullptr);
    e->cap_epoch.assign(n, -1);
    e->cap_phase.assign(n, -1);
    cudaError_t r = cudaSetDevice(e->dev);
    if (r == cudaSuccess) r = cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking);
    if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
    if (r == cudaSuccess) r = cudaEventCreate(&e->t0);
    if (r == cudaSuccess) r = cudaEventCreate(&e->t1);
    for (int i = 0; i < n && r == cudaSuccess; i++) r = cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming);
    if (r == cudaSuccess) r = cudaMalloc((void **)&e->dclk, n * sizeof(chan::DevClock));
    if (r == cudaSuccess) r = cudaMallocHost((void **)&e->hclk, n * sizeof(chan::DevClock));
    if (r != cudaSuccess) {
        g_init_error = std::string("chan_ensemble_create: ") + cudaGetErrorString(r);
        chan_ensemble_free(e);
        return CHAN_ECUDA;
    }
    for (int i = 0; i < n; i++) e->m[i]->dclk = e->dclk + i;
    *out = e;
    return CHAN_OK;
}

int chan_ensemble_size(chan_ensemble *e) { return e ? (int)e->m.size() : 0; }

int chan_ensemble_block(chan_ensemble *e) { return e ? e->L : 0; }

int chan_ensemble_step(chan_ensemble *e, int32_t nsteps, int32_t *status)
{
    if (!e || nsteps < 0) return CHAN_EINVAL;
    for (chan_ctx *c : e->m) {
        if (!c->uploaded) { e->err = "member not uploaded"; return CHAN_ESTATE; }
        if (c->diag_every > 0) { e->err = "members step without the diagnostics series"; return CHAN_ESTATE; }
    }
    EK(e, cudaSetDevice(e->dev));
    int rc = join_members_to_origin(e);
    if (rc) return rc;
    int left = nsteps;
    bool timed = false;
    if (left >= e->L) {
        if (!graph_valid(e)) {
            rc = build_graph(e);
            if (rc) return rc;
        }
        for (size_t i = 0; i < e->m.size(); i++) e->hclk[i] = chan::DevClock{e->m[i]->nstep, e->m[i]->time};
        EK(e, cudaMemcpyAsync(e->dclk, e->hclk, e->m.size() * sizeof(chan::DevClock), cudaMemcpyHostToDevice,
                              e->origin));
        EK(e, cudaEventRecord(e->t0, e->origin));
        while (left >= e->L) {
            EK(e, cudaGraphLaunch(e->exec, e->origin));
            for (chan_ctx *c : e->m) enqueue_steps(c, e->L, kCountOnly);
            e->replays++;
            left -= e->L;
        }
        EK(e, cudaEventRecord(e->t1, e->origin));
        timed = true;
    }
    rc = members_wait_origin(e);
    if (rc) return rc;
    int first = CHAN_OK;
    for (size_t i = 0; i < e->m.size(); i++) {
        chan_ctx *c = e->m[i];
        int r = left > 0 ? enqueue_steps(c, left) : CHAN_OK;
        if (r == CHAN_OK) r = read_status(c, nullptr);
        if (status) status[i] = r;
        if (r != CHAN_OK && first == CHAN_OK) first = r;
    }
    // the pinned clock staging is reused by the next call: it has been read
    EK(e, cudaStreamSynchronize(e->origin));
    if (timed && e->persistent) {
        EK(e, cudaMemcpy(e->herr, e->derr, sizeof(int), cudaMemcpyDeviceToHost));
        if (*e->herr) {
            e->err = "persistent ensemble kernel: a unit waited more than a second for its member's earlier "
                     "work and the launch stopped; the members' states are undefined (upload or restore them)";
            EK(e, cudaMemset(e->derr, 0, sizeof(int)));
            if (e->exec) { cudaGraphExecDestroy(e->exec); e->exec = nullptr; }
            return CHAN_ECUDA;
        }
    }
    e->last_ms = 0.0;
    if (timed) {
        float ms = 0.f;
        EK(e, cudaEventElapsedTime(&ms, e->t0, e->t1));
        e->last_ms = ms;
    }
    return first;
}

int chan_ensemble_tune(chan_ensemble *e, int32_t reps, double *best_ms)
{
    if (!e || reps < 1) return CHAN_EINVAL;
    for (chan_ctx *c : e->m)
        if (!c->uploaded) { e->err = "member not uploaded"; return CHAN_ESTATE; }
    EK(e, cudaSetDevice(e->dev));
    const size_t n = e->m.size();
    // the wall ring and the status are the only persistent device state the
    // trial stages write: keep copies and put them back afterwards
    std::vector<double *> wsave(n, nullptr);
    std::vector<chan::DevStatus *> ssave(n, nullptr);
    std::vector<int> cur(n);
    std::vector<int> tile(n), nch(n);
    int rc = join_members_to_origin(e);
    for (size_t i = 0; i < n && rc == CHAN_OK; i++) {
        chan_ctx *c = e->m[i];
        const size_t nw = 2 * 8 * (size_t)c->plane;
        cudaError_t r = cudaMalloc((void **)&wsave[i], nw * sizeof(double));
        if (r == cudaSuccess) r = cudaMalloc((void **)&ssave[i], sizeof(chan::DevStatus));
        if (r == cudaSuccess) r = cudaMemcpyAsync(wsave[i], c->wp, nw * sizeof(double), cudaMemcpyDeviceToDevice,
                                                  e->origin);
        if (r == cudaSuccess) r = cudaMemcpyAsync(ssave[i], c->status, sizeof(chan::DevStatus),
                                                  cudaMemcpyDeviceToDevice, e->origin);
        if (r != cudaSuccess) rc = efail(e, "tune: save", r);
        cur[i] = c->cur;
        tile[i] = c->tile;
        nch[i] = c->nchunks;
    }
    // candidate shapes of one member: each tile shape at several k-chunk depths
    auto candidates = [e](const chan_ctx *c) {
        std::vector<std::pair<int, int>> v;
        const int nz = c->n3 - 2;
        const int depth[] = {4, 8, 12, 16, 24, 32, 48, 64, 96, 128, 100000};
        for (int t = 0; t < CHAN_NTILES; t++) {
            if (e->mode == CHAN_ENSEMBLE_PERSISTENT && (t == CHAN_TILE_32x4 || t == CHAN_TILE_32x16)) continue;
            int last = -1;
            for (int d : depth) {
                const int nc = std::max(1, (nz + std::min(d, nz) - 1) / std::min(d, nz));
                const int chunk = (nz + nc - 1) / nc, real = (nz + chunk - 1) / chunk;
                if (real != last) v.push_back({t, real});
                last = real;
            }
        }
        return v;
    };
    auto apply = [&](const std::vector<int> &t, const std::vector<int> &c) {
        for (size_t i = 0; i < n; i++) {
            const int r = set_launch(e->m[i], t[i], c[i]);
            if (r) { e->err = e->m[i]->err; return r; }
        }
        return (int)CHAN_OK;
    };
    float best = 0.f, ms = 0.f;
    if (rc == CHAN_OK) rc = tune_trial(e, reps, &ms);   // warm-up of the current shapes
    if (rc == CHAN_OK) rc = tune_trial(e, reps, &best);
    // 1. one shape for every member: each tile shape at each k-chunk depth
    if (rc == CHAN_OK) {
        const int depth[] = {4, 8, 12, 16, 24, 32, 48, 64, 96, 128, 100000};
        for (int t = 0; t < CHAN_NTILES && rc == CHAN_OK; t++)
            for (int d : depth) {
                if (e->mode == CHAN_ENSEMBLE_PERSISTENT && (t == CHAN_TILE_32x4 || t == CHAN_TILE_32x16))
                    continue;   // the persistent kernel runs 256-thread CTAs
                std::vector<int> tt(n, t), cc(n);
                for (size_t i = 0; i < n; i++) {
                    const int nz = e->m[i]->n3 - 2, dd = std::min(d, nz);
                    cc[i] = (nz + dd - 1) / dd;
                }
                rc = apply(tt, cc);
                if (rc == CHAN_OK) rc = tune_trial(e, reps, &ms);
                if (rc != CHAN_OK) break;
                if (ms < best) { best = ms; tile = tt; nch = cc; }
            }
    }
    // 2. one pass of per-member refinement, largest members first
    if (rc == CHAN_OK) {
        std::vector<size_t> order(n);
        for (size_t i = 0; i < n; i++) order[i] = i;
        std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return e->m[a]->vol > e->m[b]->vol; });
        for (size_t oi = 0; oi < n && rc == CHAN_OK; oi++) {
            const size_t i = order[oi];
            for (auto cand : candidates(e->m[i])) {
                if (cand.first == tile[i] && cand.second == nch[i]) continue;
                std::vector<int> tt = tile, cc = nch;
                tt[i] = cand.first;
                cc[i] = cand.second;
                rc = apply(tt, cc);
                if (rc == CHAN_OK) rc = tune_trial(e, reps, &ms);
                if (rc != CHAN_OK) break;
                if (ms < best * 0.995f) { best = ms; tile = tt; nch = cc; }
            }
        }
    }
    int ra = apply(tile, nch);
    if (rc == CHAN_OK) rc = ra;
    // restore the wall rings, statuses and buffer roles
    for (size_t i = 0; i < n; i++) {
        chan_ctx *c = e->m[i];
        if (wsave[i] && ssave[i]) {
            cudaError_t r = cudaMemcpyAsync(c->wp, wsave[i], 2 * 8 * (size_t)c->plane * sizeof(double),
                                            cudaMemcpyDeviceToDevice, e->origin);
            if (r == cudaSuccess)
                r = cudaMemcpyAsync(c->status, ssave[i], sizeof(chan::DevStatus), cudaMemcpyDeviceToDevice, e->origin);
            if (r != cudaSuccess && rc == CHAN_OK) rc = efail(e, "tune: restore", r);
        }
        c->cur = cur[i];
    }
    cudaError_t r = cudaStreamSynchronize(e->origin);
    if (r != cudaSuccess && rc == CHAN_OK) rc = efail(e, "tune: sync", r);
    for (size_t i = 0; i < n; i++) {
        if (wsave[i]) cudaFree(wsave[i]);
        if (ssave[i]) cudaFree(ssave[i]);
    }
    if (rc == CHAN_OK) {
        const int rm = members_wait_origin(e);
        if (rm) rc = rm;
    }
    if (best_ms) *best_ms = best;
    return rc;
}

int chan_ensemble_set_mode(chan_ensemble *e, int32_t mode)
{
    if (!e) return CHAN_EINVAL;
    if (mode != CHAN_ENSEMBLE_GRAPH && mode != CHAN_ENSEMBLE_PERSISTENT && mode != CHAN_ENSEMBLE_PERSISTENT_STALL_TEST) {
        e->err = "unknown ensemble mode";
        return CHAN_EINVAL;
    }
    e->stall_test = mode == CHAN_ENSEMBLE_PERSISTENT_STALL_TEST;
    e->mode = mode == CHAN_ENSEMBLE_GRAPH ? CHAN_ENSEMBLE_GRAPH : CHAN_ENSEMBLE_PERSISTENT;
    if (e->exec) { cudaGraphExecDestroy(e->exec); e->exec = nullptr; }
    return CHAN_OK;
}

int chan_ensemble_get_mode(chan_ensemble *e, int32_t *in_use, const char **fallback_reason)
{
    if (!e) return CHAN_EINVAL;
    if (in_use) *in_use = e->exec ? (e->persistent ? CHAN_ENSEMBLE_PERSISTENT : CHAN_ENSEMBLE_GRAPH) : -1;
    if (fallback_reason) *fallback_reason = e->fallback.c_str();
    return CHAN_OK;
}

int chan_ensemble_counters(chan_ensemble *e, int64_t *replays, int64_t *captures, double *last_ms)
{
    if (!e) return CHAN_EINVAL;
    if (replays) *replays = e->replays;
    if (captures) *captures = e->captures;
    if (last_ms) *last_ms = e->last_ms;
    return CHAN_OK;
}

const char *chan_ensemble_last_error(chan_ensemble *e) { return e ? e->err.c_str() : g_init_error.c_str(); }

void chan_ensemble_free(chan_ensemble *e)
{
    if (!e) return;
    cudaSetDevice(e->dev);
    if (e->origin) cudaStreamSynchronize(e->origin);
    for (chan_ctx *c : e->m)
        if (c && c->dclk >= e->dclk && c->dclk < e->dclk + e->m.size()) c->dclk = nullptr;
    if (e->exec) cudaGraphExecDestroy(e->exec);
    for (cudaEvent_t j : e->join)
        if (j) cudaEventDestroy(j);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->t0) cudaEventDestroy(e->t0);
    if (e->t1) cudaEventDestroy(e->t1);
    if (e->dclk) cudaFree(e->dclk);
    if (e->hclk) cudaFreeHost(e->hclk);
    if (e->dph) cudaFree(e->dph);
    if (e->ditems) cudaFree(e->ditems);
    if (e->dkps) cudaFree(e->dkps);
    if (e->dmaps) cudaFree(e->dmaps);
    if (e->dcnt) cudaFree(e->dcnt);
    if (e->derr) cudaFree(e->derr);
    if (e->herr) cudaFreeHost(e->herr);
    if (e->origin) cudaStreamDestroy(e->origin);
    delete e;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// closure training samples from a context's current state (chan_internal.h)
int chan_internal_sample(chan_ctx *c, float *X, float *T, long long capacity, int sx, int sy, int sz, int fw,
                         long long *added)
{
    *added = 0;
    if (!c || !X || !T || sx < 1 || sy < 1 || sz < 1 || fw < 0 || fw % 2) return CHAN_EINVAL;
    if (!c->uploaded) return CHAN_ESTATE;
    CK(c, cudaSetDevice(c->dev));
    int r = ensure_dx3(c);
    if (r) return r;
    chan::SgsSampling S{};
    S.sx = sx; S.sy = sy; S.sz = sz; S.fw = fw;
    S.i0 = 2; S.ni = (c->n1 - 3) / sx + 1;
    S.j0 = 2; S.nj = (c->n2 - 3) / sy + 1;
    S.k0 = 1 + sz; S.nk = (c->n3 - 1) / sz - 1;
    if (S.nk < 1) return CHAN_EINVAL;
    const long long n = (long long)S.ni * S.nj * S.nk;
    if (n > capacity) { c->err = "closure dataset full"; return CHAN_EINVAL; }
    S.x3 = c->dx3;
    S.X = X;
    S.T = T;
    // the state after whole steps: q[cur] in double
    chan::k_sgs_sample<<<1184, 128, 0, c->stream>>>(c->kp, c->q[c->cur], S);
    CK(c, cudaGetLastError());
    CK(c, cudaStreamSynchronize(c->stream));
    *added = n;
    return CHAN_OK;
}
