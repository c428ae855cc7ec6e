// Batched sweeps (LBM_Batch*): one kernel launch per lattice step advances
// every grid of a batch.
//
// Each launch is k_step_batch over the concatenated tiles of all grids (a
// persistent launch of a few blocks per SM striding over the tiles); the
// per-grid arguments live in device memory (two arrays, one per buffer
// parity, since consecutive steps swap source and destination), so a CUDA
// graph of a 32-step chunk (A, B, A, B, ...) is independent of the
// arguments' values and is re-used across runs as long as the batch's
// launch shape is unchanged.  Before a run the batch stream waits for
// every grid's stream; after it every grid's stream waits for the batch.
//
// Grids leaving an explicit-f state (after LBM_InitializeFlow or a
// geometry edit) first take their priming steps through their own
// launcher; every grid takes the same number of such steps so that the
// batch stays in lock step.
#include <stdlib.h>
#include <string.h>

#include <new>
#include <vector>

#include "lbm_internal.h"

using namespace lbm;

struct LBMBatch {
    int count = 0;
    int storage = LBM_STORAGE_FP32;
    std::vector<LBMGrid *> grids;
    std::vector<int> lbx;                 // tile width exponent per grid
    std::vector<cudaEvent_t> grid_done;   // recorded on each grid's stream
    cudaEvent_t batch_done = nullptr;
    cudaStream_t stream = nullptr;
    BatchEntry *entries_dev = nullptr;    // [2][count]
    long long *starts_dev = nullptr;      // [count + 1]
    // pinned staging of the arguments, double-buffered: run k fills half
    // k % 2 after the copy out of it by run k - 2 has completed
    BatchEntry *entries_host[2] = {nullptr, nullptr};  // [2][count] each
    long long *starts_host[2] = {nullptr, nullptr};    // [count + 1] each
    cudaEvent_t copied[2] = {nullptr, nullptr};
    bool copy_pending[2] = {false, false};
    int runs = 0;
    long long blocks = 0;                 // tiles of one step (all grids)
    int set = BATCH_SET_ALL;
    int minb = 4;                         // resident blocks per SM the kernel is built for
    unsigned persist = 0;                 // persistent blocks of a full launch
    cudaGraphExec_t graph = nullptr;
    long long graph_blocks = -1;
    int graph_set = -1;
};

namespace {

constexpr int kChunk = 32;  // even: buffer parity repeats after a replay

GridImpl *impl(LBMGrid *g) { return static_cast<GridImpl *>(g->impl); }

int choose_set(const LBMBatch &b) {
    unsigned used = 0;
    for (LBMGrid *g : b.grids) used |= 1u << (grid_op(g) * 2 + (g->useSmagorinsky == 1));
    for (int s = BATCH_SET_BGK; s <= BATCH_SET_MRT_SMAG; s++)
        if (used == batch_set_mask(s)) return s;
    if ((used & ~batch_set_mask(BATCH_SET_BGK_REG)) == 0) return BATCH_SET_BGK_REG;
    return BATCH_SET_ALL;
}

BatchEntry make_entry(LBMGrid *g, int lbx, const void *src, void *dst, const float in[3]) {
    BatchEntry e{};
    e.a = grid_step_args(g, in[0], in[1], in[2]);
    e.a.src = src;
    e.a.dst = dst;
    e.a.periodic = impl(g)->stream_periodic;
    e.combo = grid_op(g) * 2 + (g->useSmagorinsky == 1);
    e.lbx = lbx;
    const int bx = 1 << lbx, by = 256 >> lbx;
    e.tiles_x = (impl(g)->nx + bx - 1) / bx;
    e.tiles_y = (impl(g)->ny + by - 1) / by;
    return e;
}

long long tiles_of(const BatchEntry &e, int nz) { return (long long)e.tiles_x * e.tiles_y * nz; }

void drop_graph(LBMBatch &b) {
    if (b.graph) {
        cudaGraphExecDestroy(b.graph);
        b.graph = nullptr;
    }
}

bool fail(LBMGrid *any, cudaError_t e) { return !grid_ok(any, e); }

unsigned persist_blocks(const LBMBatch &b) {
    return (unsigned)(b.blocks < (long long)b.persist ? b.blocks : (long long)b.persist);
}

}  // namespace

extern "C" {

LBMBatch *LBM_BatchCreate(LBMGrid **grids, int count) {
    if (!grids || count <= 0) return nullptr;
    int storage = -1;
    for (int i = 0; i < count; i++) {
        LBMGrid *g = grids[i];
        if (!g || !g->impl || !impl(g)->initialized || g->arithmetic != LBM_ARITH_EXACT)
            return nullptr;
        if (storage < 0) storage = g->storage;
        if (g->storage != storage) return nullptr;
        for (int j = 0; j < i; j++)
            if (grids[j] == g) return nullptr;  // a grid may appear once
    }
    LBMBatch *b = new (std::nothrow) LBMBatch();
    if (!b) return nullptr;
    b->count = count;
    b->storage = storage;
    b->grids.assign(grids, grids + count);
    b->lbx.assign(count, 5);  // 32 x 8 tiles, the single-grid default
    b->grid_done.assign(count, nullptr);
    // persistent launch: minb blocks per SM (LBM_BATCH_MINB=3 trades
    // occupancy for registers)
    const char *menv = getenv("LBM_BATCH_MINB");
    b->minb = (menv && atoi(menv) == 3) ? 3 : 4;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        sms <= 0) {
        delete b;
        return nullptr;
    }
    b->persist = (unsigned)(sms * b->minb);
    bool good = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess;
    good = good && cudaEventCreateWithFlags(&b->batch_done, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; good && i < count; i++)
        good = cudaEventCreateWithFlags(&b->grid_done[i], cudaEventDisableTiming) == cudaSuccess;
    good = good && cudaMalloc(&b->entries_dev, sizeof(BatchEntry) * 2 * count) == cudaSuccess;
    good = good && cudaMalloc(&b->starts_dev, sizeof(long long) * (count + 1)) == cudaSuccess;
    for (int h = 0; h < 2; h++) {
        good = good &&
               cudaMallocHost(&b->entries_host[h], sizeof(BatchEntry) * 2 * count) == cudaSuccess;
        good = good &&
               cudaMallocHost(&b->starts_host[h], sizeof(long long) * (count + 1)) == cudaSuccess;
        good = good && cudaEventCreateWithFlags(&b->copied[h], cudaEventDisableTiming) == cudaSuccess;
    }
    if (!good) {
        LBM_BatchFree(b);
        return nullptr;
    }
    return b;
}

void LBM_BatchFree(LBMBatch *b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(*b);
    for (cudaEvent_t e : b->grid_done)
        if (e) cudaEventDestroy(e);
    if (b->batch_done) cudaEventDestroy(b->batch_done);
    cudaFree(b->entries_dev);
    cudaFree(b->starts_dev);
    for (int h = 0; h < 2; h++) {
        cudaFreeHost(b->entries_host[h]);
        cudaFreeHost(b->starts_host[h]);
        if (b->copied[h]) cudaEventDestroy(b->copied[h]);
    }
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int LBM_BatchRun(LBMBatch *b, int nSteps, const float *inlet) {
    if (!b || !inlet || nSteps < 0) return LBM_ERR_INVALID_ARGUMENT;
    if (nSteps == 0) return LBM_OK;
    const int n = b->count;
    LBMGrid *g0 = b->grids[0];
    // priming: every grid takes as many solo steps as the neediest one
    int prime = 0;
    for (LBMGrid *g : b->grids) {
        GridImpl &I = *impl(g);
        if (g->arithmetic != LBM_ARITH_EXACT || g->storage != b->storage) {
            g->lastError = LBM_ERR_UNSUPPORTED;
            return LBM_ERR_UNSUPPORTED;
        }
        const int need = (I.fbuf >= 0 ? 1 : 0) +
                         ((I.fbuf >= 0 ? g->periodicYZ : I.stream_periodic) != g->periodicYZ);
        if (need > prime) prime = need;
    }
    if (prime > nSteps) prime = nSteps;
    for (int k = 0; k < prime; k++)
        for (int i = 0; i < n; i++)
            if (!grid_enqueue_step(b->grids[i], inlet[3 * i], inlet[3 * i + 1], inlet[3 * i + 2]))
                return b->grids[i]->lastError;
    const int steps = nSteps - prime;
    if (steps == 0) return LBM_OK;

    // arguments of both parities, tile offsets, launch shape
    const int h = b->runs & 1;
    if (b->copy_pending[h] && fail(g0, cudaEventSynchronize(b->copied[h]))) return LBM_ERR_CUDA;
    b->copy_pending[h] = false;
    BatchEntry *eh = b->entries_host[h];
    long long *sh = b->starts_host[h];
    long long total = 0;
    for (int i = 0; i < n; i++) {
        LBMGrid *g = b->grids[i];
        GridImpl &I = *impl(g);
        if (I.fbuf >= 0 || I.stream_periodic != g->periodicYZ) return LBM_ERR_CUDA;
        const float *in = inlet + 3 * i;
        eh[i] = make_entry(g, b->lbx[i], I.pop[I.gbuf], I.pop[1 - I.gbuf], in);
        eh[n + i] = make_entry(g, b->lbx[i], I.pop[1 - I.gbuf], I.pop[I.gbuf], in);
        sh[i] = total;
        total += tiles_of(eh[i], I.nz);
    }
    sh[n] = total;
    if (total > 0x7fffffffLL) return LBM_ERR_INVALID_ARGUMENT;
    b->blocks = total;
    b->set = choose_set(*b);

    // the batch waits for every grid's queued work
    for (int i = 0; i < n; i++) {
        if (fail(b->grids[i], cudaEventRecord(b->grid_done[i], impl(b->grids[i])->stream)))
            return LBM_ERR_CUDA;
        if (fail(b->grids[i], cudaStreamWaitEvent(b->stream, b->grid_done[i], 0)))
            return LBM_ERR_CUDA;
    }
    if (fail(g0, cudaMemcpyAsync(b->entries_dev, eh, sizeof(BatchEntry) * 2 * n,
                                 cudaMemcpyHostToDevice, b->stream)) ||
        fail(g0, cudaMemcpyAsync(b->starts_dev, sh, sizeof(long long) * (n + 1),
                                 cudaMemcpyHostToDevice, b->stream)) ||
        fail(g0, cudaEventRecord(b->copied[h], b->stream)))
        return LBM_ERR_CUDA;
    b->copy_pending[h] = true;
    b->runs++;

    const BatchEntry *ea = b->entries_dev, *eb = b->entries_dev + n;
    int left = steps;
    if (left >= kChunk) {
        if (!b->graph || b->graph_blocks != total || b->graph_set != b->set) {
            drop_graph(*b);
            cudaGraph_t graph = nullptr;
            bool good = !fail(g0, cudaStreamBeginCapture(b->stream,
                                                         cudaStreamCaptureModeThreadLocal));
            for (int k = 0; good && k < kChunk; k++)
                good = !fail(g0, launch_step_batch(b->storage, (k & 1) ? eb : ea, b->starts_dev,
                                                   n, total, b->set, b->minb, persist_blocks(*b),
                                                   b->stream));
            const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
            good = good && !fail(g0, e);
            cudaGraphExec_t exec = nullptr;
            if (good) good = !fail(g0, cudaGraphInstantiate(&exec, graph, 0));
            if (graph) cudaGraphDestroy(graph);
            if (!good) return LBM_ERR_CUDA;
            b->graph = exec;
            b->graph_blocks = total;
            b->graph_set = b->set;
        }
        while (left >= kChunk) {
            if (fail(g0, cudaGraphLaunch(b->graph, b->stream))) return LBM_ERR_CUDA;
            left -= kChunk;
        }
    }
    for (int k = 0; k < left; k++)
        if (fail(g0, launch_step_batch(b->storage, (k & 1) ? eb : ea, b->starts_dev, n, total,
                                       b->set, b->minb, persist_blocks(*b), b->stream)))
            return LBM_ERR_CUDA;

    // every grid's later work waits for the batch
    if (fail(g0, cudaEventRecord(b->batch_done, b->stream))) return LBM_ERR_CUDA;
    for (int i = 0; i < n; i++) {
        LBMGrid *g = b->grids[i];
        if (fail(g, cudaStreamWaitEvent(impl(g)->stream, b->batch_done, 0))) return LBM_ERR_CUDA;
        grid_note_fused_steps(g, steps, inlet[3 * i], inlet[3 * i + 1], inlet[3 * i + 2]);
    }
    return LBM_OK;
}

int LBM_BatchAutotune(LBMBatch *b, int trialLaunches) {
    if (!b || trialLaunches <= 0) return LBM_ERR_INVALID_ARGUMENT;
    LBMGrid *g0 = b->grids[0];
    // scratch destination large enough for the largest grid, and a guard
    // counter nobody reads
    long long nmax = 0;
    for (LBMGrid *g : b->grids) nmax = impl(g)->n > nmax ? impl(g)->n : nmax;
    void *scratch = nullptr;
    unsigned long long *guard = nullptr;
    BatchEntry *ent = nullptr;
    long long *st = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    int rc = LBM_OK;
    bool good = !fail(g0, cudaMalloc(&scratch, (size_t)nmax * 19 * impl(g0)->elem)) &&
                !fail(g0, cudaMalloc(&guard, sizeof(unsigned long long))) &&
                !fail(g0, cudaMalloc(&ent, sizeof(BatchEntry))) &&
                !fail(g0, cudaMalloc(&st, 2 * sizeof(long long))) &&
                !fail(g0, cudaEventCreate(&t0)) && !fail(g0, cudaEventCreate(&t1));
    for (int i = 0; i < b->count; i++)
        good = good && !fail(b->grids[i], cudaStreamSynchronize(impl(b->grids[i])->stream));
    good = good && !fail(g0, cudaStreamSynchronize(b->stream));
    for (int i = 0; good && i < b->count; i++) {
        LBMGrid *g = b->grids[i];
        GridImpl &I = *impl(g);
        const void *src = I.fbuf >= 0 ? I.pop[I.fbuf] : I.pop[I.gbuf];
        const float in[3] = {I.vin_inlet[0], I.vin_inlet[1], I.vin_inlet[2]};
        float best = 1e30f;
        int best_lbx = b->lbx[i];
        for (int lbx = 5; good && lbx <= 8; lbx++) {
            BatchEntry e = make_entry(g, lbx, src, scratch, in);
            e.a.guard = guard;
            const long long starts[2] = {0, tiles_of(e, I.nz)};
            const unsigned bit = 1u << e.combo;
            int set = BATCH_SET_ALL;
            for (int s = BATCH_SET_BGK; s <= BATCH_SET_MRT_SMAG; s++)
                if (bit == batch_set_mask(s)) set = s;
            good = !fail(g, cudaMemcpyAsync(ent, &e, sizeof(e), cudaMemcpyHostToDevice,
                                            b->stream)) &&
                   !fail(g, cudaMemcpyAsync(st, starts, sizeof(starts), cudaMemcpyHostToDevice,
                                            b->stream)) &&
                   !fail(g, cudaStreamSynchronize(b->stream));
            // one untimed launch, then the timed ones
            const unsigned pb = (unsigned)(starts[1] < (long long)b->persist ? starts[1]
                                                                               : b->persist);
            good = good && !fail(g, launch_step_batch(b->storage, ent, st, 1, starts[1], set,
                                                      b->minb, pb, b->stream));
            good = good && !fail(g, cudaEventRecord(t0, b->stream));
            for (int k = 0; good && k < trialLaunches; k++)
                good = !fail(g, launch_step_batch(b->storage, ent, st, 1, starts[1], set,
                                                  b->minb, pb, b->stream));
            good = good && !fail(g, cudaEventRecord(t1, b->stream)) &&
                   !fail(g, cudaEventSynchronize(t1));
            float ms = 0;
            good = good && !fail(g, cudaEventElapsedTime(&ms, t0, t1));
            // a wider tile must be at least 2 % faster to replace a narrower one
            if (good && ms < best * 0.98f) {
                best = ms;
                best_lbx = lbx;
            }
        }
        if (good && best_lbx != b->lbx[i]) {
            b->lbx[i] = best_lbx;
            drop_graph(*b);
        }
    }
    if (!good) rc = LBM_ERR_CUDA;
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(scratch);
    cudaFree(guard);
    cudaFree(ent);
    cudaFree(st);
    return rc;
}

int LBM_BatchGetTile(LBMBatch *b, int index, int *tileX, int *tileY) {
    if (!b || index < 0 || index >= b->count || !tileX || !tileY) return LBM_ERR_INVALID_ARGUMENT;
    *tileX = 1 << b->lbx[index];
    *tileY = 256 >> b->lbx[index];
    return LBM_OK;
}

int LBM_BatchSetTile(LBMBatch *b, int index, int tileX) {
    if (!b || index < 0 || index >= b->count) return LBM_ERR_INVALID_ARGUMENT;
    int lbx = -1;
    for (int k = 5; k <= 8; k++)
        if (tileX == (1 << k)) lbx = k;
    if (lbx < 0) return LBM_ERR_INVALID_ARGUMENT;
    if (b->lbx[index] != lbx) drop_graph(*b);
    b->lbx[index] = lbx;
    return LBM_OK;
}

long long LBM_BatchTilesPerStep(LBMBatch *b) {
    if (!b) return 0;
    long long total = 0;
    for (int i = 0; i < b->count; i++) {
        const int bx = 1 << b->lbx[i], by = 256 >> b->lbx[i];
        const GridImpl &I = *impl(b->grids[i]);
        total += (long long)((I.nx + bx - 1) / bx) * ((I.ny + by - 1) / by) * I.nz;
    }
    return total;
}

void *LBM_BatchGetStream(LBMBatch *b) { return b ? (void *)b->stream : nullptr; }

}  // extern "C"
