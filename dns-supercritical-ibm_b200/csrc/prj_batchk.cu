// prj_batchk.cu -- many FP64 Poisson solves of uneven sizes in one persistent kernel.
//
// A batch of independent solves (the reference solves one grid per run and plans it
// once, poisson_solver_multigpu.f90:77-129; here every case keeps its own plan) is a
// list of work items (case, stage, tiles).  The three stages of a solve are the forward
// x transform (tiles of tz x-rows of one y plane), the z solve of one x wavenumber (z
// FFT, both Thomas sweeps and inverse z FFT: k_zline's tile), and the inverse x
// transform; an x item is a run of up to 16 tiles of one case, a z item one wavenumber.
// The host orders the items stage-major (every case's forward x items, then every case's
// z items, then the inverse x items), the largest tiles first within a stage, and one
// launch of k_batch runs them all:
//
//   a CTA takes the next item index from a global counter (atomicAdd), waits until the
//   case's previous stage has completed all its tiles (a per-case, per-stage counter,
//   read with acquire semantics), runs the item's tiles with the same device functions as
//   the per-case kernels (xfft_tiles.cuh, zline_tiles.cuh), and counts them done
//   (release);
//   items are taken in order, and an item depends only on items before it, all of which
//   are held by running CTAs that wait only on earlier items, so the queue cannot
//   deadlock, whatever number of CTAs is resident;
//   every wait is bounded (a clock budget): a CTA that gives up raises the batch's
//   error word, counts its tiles done without running them (so later waits end too) and
//   continues; prj_batch_check_error reports PRJ_ERR_TIMEOUT.
//
// The tiles run the per-case kernels' code on the same elements, so every case's P
// equals its own prj_poisson_fp64 bit for bit (the z solve of k_zline is bitwise that of
// the split z kernels).  One launch replaces ncases x 3 to 5 small kernels, their launch
// gaps and their tails, and the fused z solve moves the spectrum through HBM four times
// where the split kernels move it eight.  Every staged copy (x tiles' inputs, z tiles'
// rows) is a TMA copy completed on an mbarrier; the tensor maps live in the case array
// (global memory), where the TMA unit reads them.  Counters are reset by a memset issued
// with the launch, so the pair can be captured in a CUDA graph.
#include <algorithm>
#include <array>
#include <vector>

#include "prj_internal.h"
#include "tma_util.cuh"
#include "xfft_tiles.cuh"
#include "zline_tiles.cuh"

namespace prj {

// stages of one solve
enum BatchStage { kBFwdX = 0, kBZLine = 1, kBBwdX = 2, kBNumStages = 3 };

struct __align__(64) BatchCaseDev {
    CUtensorMap zl_tmap;  // row copies of its z solves (read from global memory by the TMA unit)
    CUtensorMap x_tmap;   // spectrum copies of its inverse x tiles: {2 nz doubles, nh, ny}, box {2 tz, xbox_k, 1}
    XArgs x;          // forward (source P) and inverse (P out) x transforms of the case
    ZLineArgs zl;     // its z solves (one tile per x wavenumber)
    int xplan, zplan; // index of the x (m = nx/2) and z (nz) pass plans in PRJ_BATCH_PLANS
    int ntz;          // x tiles per y plane
    int soff;         // byte offset in shared memory of the x tiles' staged input (before 128-byte alignment)
    int sbytes;       // its bytes (xboxes spectrum boxes of xbox_k x tz values; the forward's rows fit)
    int xbox_k, xboxes;
    int tiles[kBNumStages];
};

// one work item: tiles tile0 .. tile0+count-1 of one stage of one case
struct BatchSeg {
    int case_id, stage, tile0, count;
};

namespace {

// plans the persistent kernel dispatches, indexed: the pass plans up to 256 points in
// every compiled radix order (fft_pass.cuh PRJ_PASS_PLANS and PRJ_PASS_ALTS)
#define PRJ_BATCH_PLANS(X) \
    X(0, 16, 4, 4)         \
    X(1, 24, 6, 4)         \
    X(2, 32, 8, 4)         \
    X(3, 48, 6, 8)         \
    X(4, 64, 8, 8)         \
    X(5, 96, 2, 6, 8)      \
    X(6, 128, 4, 4, 8)     \
    X(7, 192, 3, 8, 8)     \
    X(8, 256, 8, 4, 8)     \
    X(9, 64, 4, 4, 4)      \
    X(10, 96, 8, 6, 2)     \
    X(11, 128, 8, 8, 2)    \
    X(12, 192, 6, 4, 8)    \
    X(13, 256, 4, 8, 8)    \
    X(14, 256, 8, 8, 4)

constexpr int kBatchThreads = kPassThreads;
#ifndef PRJ_BATCH_MINB
#define PRJ_BATCH_MINB 6
#endif
// resident CTAs per SM the register allocation is held to (6: at most 80 registers per
// thread, the per-case x kernels' own allocation)
constexpr int kBatchMinBlocks = PRJ_BATCH_MINB;

// Every (stage, plan) tile is its own non-inlined function: inlined into one switch, the
// thirty plan variants' butterflies shared one register allocation and spilled (2 KB of
// stack per thread); as calls, each tile function is allocated on its own, as in its
// per-case kernel.
//
// The x stages run an item's tiles as a pipeline (x_tiles_tma, xfft_tiles.cuh): the next
// tile's input is copied into shared memory by the TMA unit while the current tile
// computes, so a CTA keeps loads in flight through its FFT passes and stores instead of
// one round trip per tile; the z tiles stream their planes through zline_tile's ring.
template <class PL, bool FWD>
__device__ __forceinline__ void run_x_tiles(const BatchCaseDev& c, const CUtensorMap* xmap, int t0, int count,
                                            unsigned char* sm, int* err) {
    x_tiles_tma<PL, FWD, false>(c.x, xmap, c.ntz, c.xboxes, c.xbox_k, sm, c.soff, c.sbytes, t0, 1, t0 + count, err);
}
template <class PL>
__device__ __noinline__ void run_x_fwd_tiles(const BatchCaseDev& c, const CUtensorMap* xmap, int t0, int count,
                                             unsigned char* sm, int* err) {
    run_x_tiles<PL, true>(c, xmap, t0, count, sm, err);
}
template <class PL>
__device__ __noinline__ void run_x_bwd_tiles(const BatchCaseDev& c, const CUtensorMap* xmap, int t0, int count,
                                             unsigned char* sm, int* err) {
    run_x_tiles<PL, false>(c, xmap, t0, count, sm, err);
}
// the z solve of one wavenumber: ring of kZlStages stages of c.zl.yb planes, lines
// spread over the CTA's threads
constexpr int kZlStages = 2;
__host__ __device__ constexpr int batch_lpt(int n) { return (n + kBatchThreads - 1) / kBatchThreads; }
template <class PL>
__device__ __noinline__ void tile_zline(const BatchCaseDev& c, const CUtensorMap* tmap, int kx, unsigned char* sm) {
    zline_tile<PL, kZlStages, batch_lpt(PL::n), kBatchThreads>(c.zl, tmap, kx, sm);
}

__device__ __forceinline__ void run_x_fwd(const BatchCaseDev& c, const CUtensorMap* xmap, int t0, int count,
                                          unsigned char* sm, int* err) {
    switch (c.xplan) {
#define PRJ_BX(I, N, ...) \
    case I: run_x_fwd_tiles<PassList<__VA_ARGS__>>(c, xmap, t0, count, sm, err); break;
        PRJ_BATCH_PLANS(PRJ_BX)
#undef PRJ_BX
    default: break;
    }
}

__device__ __forceinline__ void run_x_bwd(const BatchCaseDev& c, const CUtensorMap* xmap, int t0, int count,
                                          unsigned char* sm, int* err) {
    switch (c.xplan) {
#define PRJ_BX(I, N, ...) \
    case I: run_x_bwd_tiles<PassList<__VA_ARGS__>>(c, xmap, t0, count, sm, err); break;
        PRJ_BATCH_PLANS(PRJ_BX)
#undef PRJ_BX
    default: break;
    }
}

__device__ __forceinline__ void run_zline(const BatchCaseDev& c, const CUtensorMap* tmap, int kx, unsigned char* sm) {
    switch (c.zplan) {
#define PRJ_BZ(I, N, ...) \
    case I: tile_zline<PassList<__VA_ARGS__>>(c, tmap, kx, sm); break;
        PRJ_BATCH_PLANS(PRJ_BZ)
#undef PRJ_BZ
    default: break;
    }
}

__global__ void __launch_bounds__(kBatchThreads, kBatchMinBlocks)
    k_batch(const BatchCaseDev* __restrict__ cases, const BatchSeg* __restrict__ segs, int nseg,
            unsigned long long* counter, int* done, int* err) {
    extern __shared__ __align__(128) unsigned char bsm[];
    __shared__ BatchSeg s_seg;
    __shared__ int s_skip;
    // the current case's arguments, copied once per change of case (the items of one case
    // and stage come in runs) so that the tile functions read them from shared memory
    __shared__ __align__(64) BatchCaseDev s_case;
    int loaded = -1;
    for (;;) {
        if (threadIdx.x == 0) {
            const long long it = (long long)atomicAdd(counter, 1ull);
            BatchSeg g{-1, 0, 0, 0};
            int skip = 0;
            if (it < nseg) {
                g = segs[it];
                if (g.stage > 0) {
                    const int need = cases[g.case_id].tiles[g.stage - 1];
                    const volatile int* d = done + g.case_id * kBNumStages + g.stage - 1;
                    const long long t0 = clock64();
                    while (*d < need) {
                        if (clock64() - t0 > kWaitBudgetCycles) {
                            atomicExch(err, 4);
                            skip = 1;
                            break;
                        }
                        __nanosleep(128);
                    }
                    __threadfence();  // acquire: the previous stage's results before this item's reads
                    fence_proxy_async_global();  // ... and before the tensor-map copies this thread issues
                }
            }
            s_seg = g;
            s_skip = skip;
        }
        __syncthreads();
        const BatchSeg g = s_seg;
        if (g.case_id < 0) break;
        if (g.case_id != loaded) {
            static_assert(sizeof(BatchCaseDev) % 16 == 0, "16-byte copies");
            const int4* src = reinterpret_cast<const int4*>(cases + g.case_id);
            int4* dst = reinterpret_cast<int4*>(&s_case);
            for (int w = threadIdx.x; w < (int)(sizeof(BatchCaseDev) / 16); w += blockDim.x) dst[w] = src[w];
            __syncthreads();
            loaded = g.case_id;
        }
        const BatchCaseDev& c = s_case;
        if (!s_skip) {
            switch (g.stage) {
            case kBFwdX: run_x_fwd(c, &cases[g.case_id].x_tmap, g.tile0, g.count, bsm, err); break;
            case kBBwdX: run_x_bwd(c, &cases[g.case_id].x_tmap, g.tile0, g.count, bsm, err); break;
            default:
                for (int kx = g.tile0; kx < g.tile0 + g.count; kx++) {
                    run_zline(c, &cases[g.case_id].zl_tmap, kx, bsm);
                    __syncthreads();  // bsm free for the next tile
                }
                break;
            }
        }
        fence_proxy_async_global();  // this thread's stores, for later tensor-map reads of other CTAs
        __syncthreads();  // every thread's stores of the item
        if (threadIdx.x == 0) {
            __threadfence();  // release: the item's stores before its count
            atomicAdd(done + g.case_id * kBNumStages + g.stage, g.count);
        }
    }
}

// shared memory of an x tile's staged input (the inverse's boxes of tz values; the forward's
// tz rows of m fit) with 128 bytes of alignment slack and the mbarrier
size_t x_stage_bytes(int m, int tz) { return 128 + (size_t)x_boxes(m) * x_box_k(m) * tz * sizeof(double2) + 16; }
// dynamic shared memory of a tile with its staged input: six CTAs of 128 threads per SM
// (228 KB per SM, 1 KB reserved and ~2 KB static per CTA)
constexpr size_t kStagedBytes = 34 * 1024 + 512;

int batch_plan_index(int n, const DifDev& f) {
#define PRJ_BI(I, N, ...) \
    if (n == N && same_radices<PassList<__VA_ARGS__>>(f)) return I;
    PRJ_BATCH_PLANS(PRJ_BI)
#undef PRJ_BI
    return -1;
}

}  // namespace

bool batchk_supported(const prj_plan* pl) {
    return pl->use_pass && pl->fx64.even && pl->xd.ok && pl->zd.ok && pl->kz_of_slot && pl->t.pivc &&
           batch_plan_index(pl->fx64.m, pl->xd.f) >= 0 && batch_plan_index(pl->g.nz, pl->zd.f) >= 0 &&
           pl->kxs == pl->g.nxh;
}

cudaError_t batchk_build(prj_plan* const* plans, double* const* d_P, int ncases, BatchKernel* out) {
    std::vector<BatchCaseDev> cs((size_t)ncases);
    std::vector<std::array<long long, kBNumStages>> work((size_t)ncases);
    size_t smem = 0;
    for (int i = 0; i < ncases; i++) {
        const prj_plan* pl = plans[i];
        const Geometry& g = pl->g;
        BatchCaseDev& c = cs[i];
        c.x = batch_x_args(pl, d_P[i]);
        c.zl = zline_args(pl);
        // x tile shapes within the per-case kernels' default shared-memory budgets and, with
        // their staged input, within kStagedBytes, so six CTAs fit per SM whatever the
        // plans' own tuning; a tile's shape does not change its results
        const int m = pl->fx64.m;
        c.x.tz = std::min(c.x.tz, choose_tz_xp(m));
        while (c.x.tz > 1 && pass_x_smem(m, c.x.tz) + x_stage_bytes(m, c.x.tz) > kStagedBytes) c.x.tz /= 2;
        c.soff = (int)pass_x_smem(m, c.x.tz);
        c.xboxes = x_boxes(m);
        c.xbox_k = x_box_k(m);
        c.sbytes = c.xboxes * c.xbox_k * c.x.tz * (int)sizeof(double2);
        {
            const uint64_t dims[3] = {2 * (uint64_t)g.nz, (uint64_t)g.nxh, (uint64_t)g.ny};
            const uint64_t strides[2] = {(uint64_t)g.nz * 16, (uint64_t)g.nxh * (uint64_t)g.nz * 16};
            const uint32_t box[3] = {2 * (uint32_t)c.x.tz, (uint32_t)c.xbox_k, 1};
            if (2 * c.x.tz > 256 || !tmap_encode_f64(&c.x_tmap, pl->spec, 3, dims, strides, box)) return cudaErrorNotSupported;
        }
        // planes per stage of the z solve's ring: up to 8 within kStagedBytes
        c.zl.yb = std::min(8, g.ny);
        while (c.zl.yb > 1 && zline_smem(g.nz, g.mzp, c.zl.yb, kZlStages) > kStagedBytes) c.zl.yb--;
        if (!zline_tmap(&c.zl_tmap, pl->spec, g.nz, g.nxh, g.ny, c.zl.yb)) return cudaErrorNotSupported;
        c.xplan = batch_plan_index(pl->fx64.m, pl->xd.f);
        c.zplan = batch_plan_index(g.nz, pl->zd.f);
        c.ntz = (g.nz + c.x.tz - 1) / c.x.tz;
        c.tiles[kBFwdX] = c.tiles[kBBwdX] = c.ntz * g.ny;
        c.tiles[kBZLine] = g.nxh;
        // work of one tile of each stage (points), the order key within a stage
        work[i][kBFwdX] = work[i][kBBwdX] = (long long)c.x.tz * g.nx;
        work[i][kBZLine] = (long long)g.ny * g.nz;
        smem = std::max(smem, pass_x_smem(m, c.x.tz) + x_stage_bytes(m, c.x.tz));
        smem = std::max(smem, zline_smem(g.nz, g.mzp, c.zl.yb, kZlStages));
    }
    // stage-major order; within a stage the cases with the largest tiles first (the longest
    // z solves start first, so the stage's tail is short); each x stage of a case cut into
    // items of up to 16 tiles (about 64 items per stage where it has that many tiles), so
    // one counter increment and one load start several tiles; a z item is one wavenumber
    std::vector<int> order((size_t)ncases);
    for (int i = 0; i < ncases; i++) order[i] = i;
    std::vector<BatchSeg> segs;
    long long tiles_total = 0;
    for (int s = 0; s < kBNumStages; s++) {
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return work[a][s] != work[b][s] ? work[a][s] > work[b][s] : cs[a].tiles[s] > cs[b].tiles[s];
        });
        for (int i : order) {
            const int T = cs[i].tiles[s];
            const int chunk = s == kBZLine ? 1 : std::max(1, std::min(16, T / 64));
            for (int t0 = 0; t0 < T; t0 += chunk) segs.push_back(BatchSeg{i, s, t0, std::min(chunk, T - t0)});
            tiles_total += T;
        }
    }
    const long long items = (long long)segs.size();
    if (smem > (size_t)200 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 1));
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch, kBatchThreads, smem)) != cudaSuccess) return e;
    if (per < 1) return cudaErrorInvalidConfiguration;
    out->grid = (int)std::min<long long>((long long)per * sms, items);
    out->smem = smem;
    out->nseg = (int)segs.size();
    out->nitems = items;
    out->ntiles = tiles_total;
    out->ncases = ncases;
    const size_t cb = cs.size() * sizeof(BatchCaseDev), sb = segs.size() * sizeof(BatchSeg);
    const size_t wb = sizeof(unsigned long long) + (size_t)ncases * kBNumStages * sizeof(int) + sizeof(int);
    if ((e = cudaMalloc(&out->d_cases, cb)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&out->d_segs, sb)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&out->d_work, wb)) != cudaSuccess) return e;
    out->work_bytes = wb - sizeof(int);  // the error word after the counters is cleared by its check
    int* errw = reinterpret_cast<int*>(static_cast<unsigned char*>(out->d_work) + out->work_bytes);
    for (BatchCaseDev& c : cs) c.zl.err = errw;  // a z tile's wait that gives up raises the batch's word
    static_assert(sizeof(BatchCaseDev) % 64 == 0, "tensor maps 64-byte aligned in the case array");
    if ((e = cudaMemcpy(out->d_cases, cs.data(), cb, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if ((e = cudaMemcpy(out->d_segs, segs.data(), sb, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    return cudaMemset(out->d_work, 0, wb);
}

cudaError_t batchk_launch(const BatchKernel& k, cudaStream_t st) {
    unsigned char* w = static_cast<unsigned char*>(k.d_work);
    cudaError_t e = cudaMemsetAsync(w, 0, k.work_bytes, st);
    if (e != cudaSuccess) return e;
    unsigned long long* counter = reinterpret_cast<unsigned long long*>(w);
    int* done = reinterpret_cast<int*>(w + sizeof(unsigned long long));
    int* err = done + (size_t)k.ncases * kBNumStages;
    k_batch<<<k.grid, kBatchThreads, k.smem, st>>>(static_cast<const BatchCaseDev*>(k.d_cases),
                                                   static_cast<const BatchSeg*>(k.d_segs), k.nseg, counter, done,
                                                   err);
    return cudaGetLastError();
}

int* batchk_err_word(const BatchKernel& k) {
    return reinterpret_cast<int*>(static_cast<unsigned char*>(k.d_work) + k.work_bytes);
}

void batchk_free(BatchKernel* k) {
    if (k->d_cases) cudaFree(k->d_cases);
    if (k->d_segs) cudaFree(k->d_segs);
    if (k->d_work) cudaFree(k->d_work);
    *k = BatchKernel{};
}

}  // namespace prj
