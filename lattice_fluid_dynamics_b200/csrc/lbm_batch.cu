// Batched sweeps (LBM_Batch*): one kernel launch per lattice step advances
// up to 64 grids of one operator (a batch takes one launch per operator and
// per 64 grids).
//
// Each launch is k_step_batch over the concatenated tiles of its grids, the
// per-grid arguments passed by value in the kernel parameter (two argument
// sets, one per buffer parity, since consecutive steps swap source and
// destination).  A CUDA graph of a 32-step chunk (A, B, A, B, ...) is
// captured with those arguments and replayed while they stay the same.
// Before a run the batch stream waits for every grid's stream; after it
// every grid's stream waits for the batch.
//
// Grids leaving an explicit-f state (after LBM_InitializeFlow or a
// geometry edit) first take their priming steps through their own
// launcher; every grid takes the same number of such steps so that the
// batch stays in lock step.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
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
    // launch groups: grid indices, ordered by operator, at most
    // BATCH_LAUNCH_MAX per group; arguments of both buffer parities
    std::vector<std::vector<int>> groups;
    std::vector<BatchLaunchParams> params[2];
    std::vector<int> sets;
    // the CUDA graph of kChunk steps and the arguments it was captured with
    cudaGraphExec_t graph = nullptr;
    std::vector<BatchLaunchParams> graph_params[2];
    std::vector<int> graph_sets;
};

namespace {

constexpr int kChunk = 32;  // even: buffer parity repeats after a replay

GridImpl *impl(LBMGrid *g) { return static_cast<GridImpl *>(g->impl); }

int combo_of(LBMGrid *g) { return grid_op(g) * 2 + (g->useSmagorinsky == 1); }

int set_of(unsigned used) {
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
    e.combo = combo_of(g);
    e.lbx = lbx;
    const int bx = 1 << lbx, by = 256 >> lbx;
    e.tiles_x = (impl(g)->nx + bx - 1) / bx;
    e.tiles_y = (impl(g)->ny + by - 1) / by;
    return e;
}

// work units (tile columns of BATCH_ZB z-planes) of one grid
long long units_of(const BatchEntry &e, int nz) {
    return (long long)e.tiles_x * e.tiles_y * ((nz + BATCH_ZB - 1) / BATCH_ZB);
}

void drop_graph(LBMBatch &b) {
    if (b.graph) {
        cudaGraphExecDestroy(b.graph);
        b.graph = nullptr;
    }
}

bool fail(LBMGrid *any, cudaError_t e) { return !grid_ok(any, e); }

// one launch group per operator (each gets the kernel specialised to it),
// cut into groups of at most BATCH_LAUNCH_MAX grids
void make_groups(LBMBatch &b) {
    b.groups.clear();
    for (int c = 0; c < 6; c++) {
        std::vector<int> grp;
        for (int i = 0; i < b.count; i++)
            if (combo_of(b.grids[i]) == c) grp.push_back(i);
        for (size_t k = 0; k < grp.size(); k += BATCH_LAUNCH_MAX)
            b.groups.emplace_back(grp.begin() + k,
                                  grp.begin() + std::min(grp.size(), k + BATCH_LAUNCH_MAX));
    }
}

bool same_params(const std::vector<BatchLaunchParams> &a, const std::vector<BatchLaunchParams> &c) {
    if (a.size() != c.size()) return false;
    for (size_t i = 0; i < a.size(); i++)
        if (memcmp(&a[i], &c[i], sizeof(BatchLaunchParams)) != 0) return false;
    return true;
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
    bool good = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess;
    good = good && cudaEventCreateWithFlags(&b->batch_done, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; good && i < count; i++)
        good = cudaEventCreateWithFlags(&b->grid_done[i], cudaEventDisableTiming) == cudaSuccess;
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

    // launch arguments of both parities for every group
    make_groups(*b);
    const size_t ng = b->groups.size();
    for (int p = 0; p < 2; p++) b->params[p].assign(ng, BatchLaunchParams{});
    b->sets.assign(ng, BATCH_SET_ALL);
    for (size_t gi = 0; gi < ng; gi++) {
        const std::vector<int> &grp = b->groups[gi];
        unsigned used = 0;
        long long total = 0;
        for (size_t j = 0; j < grp.size(); j++) {
            const int i = grp[j];
            LBMGrid *g = b->grids[i];
            GridImpl &I = *impl(g);
            if (I.fbuf >= 0 || I.stream_periodic != g->periodicYZ) return LBM_ERR_CUDA;
            const float *in = inlet + 3 * i;
            b->params[0][gi].e[j] = make_entry(g, b->lbx[i], I.pop[I.gbuf], I.pop[1 - I.gbuf], in);
            b->params[1][gi].e[j] = make_entry(g, b->lbx[i], I.pop[1 - I.gbuf], I.pop[I.gbuf], in);
            b->params[0][gi].starts[j] = b->params[1][gi].starts[j] = (unsigned)total;
            total += units_of(b->params[0][gi].e[j], I.nz);
            used |= 1u << combo_of(g);
        }
        if (total > 0x7fffffffLL) return LBM_ERR_INVALID_ARGUMENT;
        for (int p = 0; p < 2; p++) {
            b->params[p][gi].starts[grp.size()] = (unsigned)total;
            b->params[p][gi].count = (int)grp.size();
        }
        b->sets[gi] = set_of(used);
    }

    // the batch waits for every grid's queued work
    for (int i = 0; i < n; i++) {
        if (fail(b->grids[i], cudaEventRecord(b->grid_done[i], impl(b->grids[i])->stream)))
            return LBM_ERR_CUDA;
        if (fail(b->grids[i], cudaStreamWaitEvent(b->stream, b->grid_done[i], 0)))
            return LBM_ERR_CUDA;
    }
    auto step = [&](int parity) {
        for (size_t gi = 0; gi < ng; gi++)
            if (fail(g0, launch_step_batch(b->storage, b->params[parity][gi], b->sets[gi],
                                           b->stream)))
                return false;
        return true;
    };
    int left = steps;
    if (left >= kChunk) {
        if (!b->graph || b->graph_sets != b->sets || !same_params(b->graph_params[0], b->params[0]) ||
            !same_params(b->graph_params[1], b->params[1])) {
            drop_graph(*b);
            cudaGraph_t graph = nullptr;
            bool good = !fail(g0, cudaStreamBeginCapture(b->stream,
                                                         cudaStreamCaptureModeThreadLocal));
            for (int k = 0; good && k < kChunk; k++) good = step(k & 1);
            const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
            good = good && !fail(g0, e);
            cudaGraphExec_t exec = nullptr;
            if (good) good = !fail(g0, cudaGraphInstantiate(&exec, graph, 0));
            if (graph) cudaGraphDestroy(graph);
            if (!good) return LBM_ERR_CUDA;
            b->graph = exec;
            b->graph_params[0] = b->params[0];
            b->graph_params[1] = b->params[1];
            b->graph_sets = b->sets;
        }
        while (left >= kChunk) {
            if (fail(g0, cudaGraphLaunch(b->graph, b->stream))) return LBM_ERR_CUDA;
            left -= kChunk;
        }
    }
    for (int k = 0; k < left; k++)
        if (!step(k & 1)) return LBM_ERR_CUDA;

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
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    bool good = !fail(g0, cudaMalloc(&scratch, (size_t)nmax * 19 * impl(g0)->elem)) &&
                !fail(g0, cudaMalloc(&guard, sizeof(unsigned long long))) &&
                !fail(g0, cudaEventCreate(&t0)) && !fail(g0, cudaEventCreate(&t1));
    for (int i = 0; i < b->count; i++)
        good = good && !fail(b->grids[i], cudaStreamSynchronize(impl(b->grids[i])->stream));
    good = good && !fail(g0, cudaStreamSynchronize(b->stream));
    BatchLaunchParams p{};
    for (int i = 0; good && i < b->count; i++) {
        LBMGrid *g = b->grids[i];
        GridImpl &I = *impl(g);
        const void *src = I.fbuf >= 0 ? I.pop[I.fbuf] : I.pop[I.gbuf];
        const float in[3] = {I.vin_inlet[0], I.vin_inlet[1], I.vin_inlet[2]};
        float best = 1e30f;
        int best_lbx = b->lbx[i];
        for (int lbx = 5; good && lbx <= 8; lbx++) {
            p.e[0] = make_entry(g, lbx, src, scratch, in);
            p.e[0].a.guard = guard;
            p.starts[0] = 0;
            p.starts[1] = (unsigned)units_of(p.e[0], I.nz);
            p.count = 1;
            const int set = set_of(1u << p.e[0].combo);
            // one untimed launch, then the timed ones
            good = !fail(g, launch_step_batch(b->storage, p, set, b->stream)) &&
                   !fail(g, cudaEventRecord(t0, b->stream));
            for (int k = 0; good && k < trialLaunches; k++)
                good = !fail(g, launch_step_batch(b->storage, p, set, b->stream));
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
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(scratch);
    cudaFree(guard);
    return good ? LBM_OK : LBM_ERR_CUDA;
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
