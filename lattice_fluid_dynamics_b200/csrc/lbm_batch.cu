// Batched sweeps (LBM_Batch*): many independent grids advanced together.
//
// Two schedules, chosen per batch by LBM_BatchAutotune from measurements:
//   fused - one kernel launch per step for up to 64 grids of one collision
//           operator: the grids' tiles concatenated, each block reading its
//           grid's entry from a table in device memory into shared memory
//           (k_step_batch_pair, two cells per thread; batches holding an
//           FP64 grid or an odd NX take the one-cell k_step_batch, whose
//           entries are in the kernel parameter);
//   graph - every grid's own fused step kernel (k_step_pair or k_step, the
//           grid's tile shape), the grids spread over a few streams that run
//           concurrently.
// Either way a 32-step chunk is captured once as a CUDA graph and replayed
// while the arguments stay the same (one graph launch per chunk), and every
// grid's populations are bit-identical to stepping it alone.  Before a run
// the batch stream waits for every grid's stream; after it every grid's
// stream waits for the batch.
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

namespace {
enum { MODE_FUSED = 0, MODE_GRAPH = 1 };
constexpr int kChunk = 32;    // even: buffer parity repeats after a replay
constexpr int kStreams = 4;   // concurrent streams of the graph schedule
}  // namespace

struct LBMBatch {
    int count = 0;
    int storage = LBM_STORAGE_FP32;
    int mode = MODE_FUSED;
    // every grid can take the paired kernels (FP32 / FP16 / BF16, even NX)
    bool pair = false;
    // the paired fused schedule's grid entries in group order: host copies,
    // what was last uploaded, and the device tables, one per buffer parity
    std::vector<BatchGridDev> tab[2];
    std::vector<BatchGridDev> tab_uploaded[2];
    BatchGridDev *dev_tab[2] = {nullptr, nullptr};
    std::vector<BatchPairParams> pparams[2];
    std::vector<BatchPairParams> graph_pparams[2];
    std::vector<LBMGrid *> grids;
    std::vector<int> lbx;                 // tile width exponent per grid
    std::vector<cudaEvent_t> grid_done;   // recorded on each grid's stream
    cudaEvent_t batch_done = nullptr;
    cudaEvent_t fork = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t side[kStreams] = {};
    cudaEvent_t side_done[kStreams] = {};
    std::vector<int> lane;                // stream of each grid (graph schedule)
    // fused schedule: launch groups (one operator, <= BATCH_LAUNCH_MAX grids)
    std::vector<std::vector<int>> groups;
    std::vector<BatchLaunchParams> params[2];
    std::vector<int> sets;
    // graph schedule: each grid's step arguments of both buffer parities
    std::vector<StepArgs> args[2];
    // the captured chunk and what it was captured with
    cudaGraphExec_t graph = nullptr;
    int graph_mode = -1;
    std::vector<BatchLaunchParams> graph_params[2];
    std::vector<int> graph_sets;
    std::vector<StepArgs> graph_args[2];
    std::vector<int> graph_lbx;
};

// the tile of a grid in cells: pair batches 2 << lbx by 128 >> lbx (lbx 5..7),
// one-cell batches 1 << lbx by 256 >> lbx (lbx 5..8)
static int tile_x_cells(const LBMBatch &b, int lbx) { return b.pair ? 2 << lbx : 1 << lbx; }
static int tile_y_cells(const LBMBatch &b, int lbx) { return b.pair ? 128 >> lbx : 256 >> lbx; }
static int lbx_min() { return 5; }
static int lbx_max(const LBMBatch &b) { return b.pair ? 7 : 8; }

namespace {

GridImpl *impl(LBMGrid *g) { return static_cast<GridImpl *>(g->impl); }

int combo_of(LBMGrid *g) { return grid_op(g) * 2 + (g->useSmagorinsky == 1); }

int set_of(unsigned used) {
    for (int s = BATCH_SET_BGK; s <= BATCH_SET_MRT_SMAG; s++)
        if (used == batch_set_mask(s)) return s;
    if ((used & ~batch_set_mask(BATCH_SET_BGK_REG)) == 0) return BATCH_SET_BGK_REG;
    return BATCH_SET_ALL;
}

StepArgs step_of(LBMGrid *g, const void *src, void *dst, const float in[3]) {
    StepArgs a = grid_step_args(g, in[0], in[1], in[2]);
    a.src = src;
    a.dst = dst;
    a.periodic = impl(g)->stream_periodic;
    return a;
}

bool same_args(const StepArgs &a, const StepArgs &b) {
    return a.src == b.src && a.dst == b.dst && a.flags == b.flags && a.slot == b.slot &&
           a.bmask == b.bmask && a.bfirst == b.bfirst && a.lq == b.lq && a.nx == b.nx &&
           a.ny == b.ny && a.nz == b.nz && a.n == b.n && a.periodic == b.periodic &&
           a.tau == b.tau && a.omega == b.omega && a.smag18 == b.smag18 &&
           a.omega_d == b.omega_d && a.smag18_d == b.smag18_d && a.inX == b.inX &&
           a.inY == b.inY && a.inZ == b.inZ && a.guard == b.guard && a.err == b.err;
}

bool same_params(const std::vector<BatchLaunchParams> &x, const std::vector<BatchLaunchParams> &y) {
    if (x.size() != y.size()) return false;
    for (size_t i = 0; i < x.size(); i++) {
        const BatchLaunchParams &a = x[i], &b = y[i];
        if (a.count != b.count) return false;
        for (int j = 0; j <= a.count; j++)
            if (a.starts[j] != b.starts[j]) return false;
        for (int j = 0; j < a.count; j++)
            if (!same_args(a.e[j].a, b.e[j].a) || a.e[j].combo != b.e[j].combo ||
                a.e[j].lbx != b.e[j].lbx || a.e[j].tiles_x != b.e[j].tiles_x ||
                a.e[j].tiles_y != b.e[j].tiles_y)
                return false;
    }
    return true;
}

bool same_pair_params(const std::vector<BatchPairParams> &x,
                      const std::vector<BatchPairParams> &y) {
    if (x.size() != y.size()) return false;
    for (size_t i = 0; i < x.size(); i++) {
        if (x[i].grids != y[i].grids || x[i].count != y[i].count) return false;
        for (int j = 0; j <= x[i].count; j++)
            if (x[i].starts[j] != y[i].starts[j]) return false;
    }
    return true;
}

bool same_arg_vec(const std::vector<StepArgs> &x, const std::vector<StepArgs> &y) {
    if (x.size() != y.size()) return false;
    for (size_t i = 0; i < x.size(); i++)
        if (!same_args(x[i], y[i])) return false;
    return true;
}

BatchEntry make_entry(LBMGrid *g, int lbx, const StepArgs &a) {
    BatchEntry e{};
    e.a = a;
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

// streams of the graph schedule: largest grids first onto the least loaded
void make_lanes(LBMBatch &b) {
    std::vector<int> order(b.count);
    for (int i = 0; i < b.count; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return impl(b.grids[x])->n > impl(b.grids[y])->n; });
    long long load[kStreams] = {0};
    b.lane.assign(b.count, 0);
    for (int i : order) {
        int best = 0;
        for (int s = 1; s < kStreams; s++)
            if (load[s] < load[best]) best = s;
        b.lane[i] = best;
        load[best] += impl(b.grids[i])->n;
    }
}

// fused launch arguments of every group for per-grid step arguments a[i]
bool build_params(LBMBatch &b, const std::vector<StepArgs> &a, std::vector<BatchLaunchParams> &out,
                  std::vector<int> &sets) {
    out.assign(b.groups.size(), BatchLaunchParams{});
    sets.assign(b.groups.size(), BATCH_SET_ALL);
    for (size_t gi = 0; gi < b.groups.size(); gi++) {
        const std::vector<int> &grp = b.groups[gi];
        unsigned used = 0;
        long long total = 0;
        for (size_t j = 0; j < grp.size(); j++) {
            const int i = grp[j];
            out[gi].e[j] = make_entry(b.grids[i], b.lbx[i], a[i]);
            out[gi].starts[j] = (unsigned)total;
            total += units_of(out[gi].e[j], impl(b.grids[i])->nz);
            used |= 1u << combo_of(b.grids[i]);
        }
        if (total > 0x7fffffffLL) return false;
        out[gi].starts[grp.size()] = (unsigned)total;
        out[gi].count = (int)grp.size();
        sets[gi] = set_of(used);
    }
    return true;
}

// the grid's fused step kernel with the batch's tile shape for it
cudaError_t grid_step(LBMBatch &b, int i, const StepArgs &a, cudaStream_t s) {
    GridImpl t = *impl(b.grids[i]);
    if (b.pair) {
        t.cpt = 2;
        t.pbx = 1 << b.lbx[i];
    } else {
        t.bx = 1 << b.lbx[i];
        t.by = 256 >> b.lbx[i];
        t.cpt = 1;
    }
    t.minb = 4;
    const int op = grid_op(b.grids[i]);
    return launch_step(t, a, true, op, b.grids[i]->useSmagorinsky == 1, false, s);
}

// `steps` steps of the whole batch in the graph schedule: forked from the
// batch stream onto the side streams, each stream stepping its grids with
// the arguments of alternating parity (a[0], a[1], a[0], ...), joined back
// at the end; grids on different streams run concurrently
bool steps_graph(LBMBatch &b, const std::vector<StepArgs> *a, int steps) {
    LBMGrid *g0 = b.grids[0];
    if (fail(g0, cudaEventRecord(b.fork, b.stream))) return false;
    for (int s = 0; s < kStreams; s++)
        if (fail(g0, cudaStreamWaitEvent(b.side[s], b.fork, 0))) return false;
    for (int k = 0; k < steps; k++)
        for (int i = 0; i < b.count; i++)
            if (fail(b.grids[i], grid_step(b, i, a[k & 1][i], b.side[b.lane[i]]))) return false;
    for (int s = 0; s < kStreams; s++)
        if (fail(g0, cudaEventRecord(b.side_done[s], b.side[s])) ||
            fail(g0, cudaStreamWaitEvent(b.stream, b.side_done[s], 0)))
            return false;
    return true;
}

bool step_fused(LBMBatch &b, const std::vector<BatchLaunchParams> &p, const std::vector<int> &sets) {
    for (size_t gi = 0; gi < p.size(); gi++)
        if (fail(b.grids[0], launch_step_batch(b.storage, p[gi], sets[gi], b.stream))) return false;
    return true;
}

BatchGridDev pair_entry(LBMBatch &b, int i, const StepArgs &a) {
    BatchGridDev e;
    memset(&e, 0, sizeof(e));  // padding too: entries are compared bytewise
    e.a = a;
    e.nz = make_float2(-0.0f, -0.0f);
    e.combo = combo_of(b.grids[i]);
    e.lbx = b.lbx[i];
    e.tiles_x = (impl(b.grids[i])->nx + tile_x_cells(b, e.lbx) - 1) / tile_x_cells(b, e.lbx);
    e.tiles_y = (impl(b.grids[i])->ny + tile_y_cells(b, e.lbx) - 1) / tile_y_cells(b, e.lbx);
    return e;
}

// The paired entries of every grid for per-grid step arguments a, in group
// order (the grids of group 0, then of group 1, ...), copied to device table
// `parity` when they differ from what it holds.
bool upload_pair_table(LBMBatch &b, const std::vector<StepArgs> &a, int parity) {
    std::vector<BatchGridDev> &t = b.tab[parity];
    t.clear();
    for (const std::vector<int> &grp : b.groups)
        for (int i : grp) t.push_back(pair_entry(b, i, a[i]));
    const size_t bytes = sizeof(BatchGridDev) * t.size();
    if (b.tab_uploaded[parity].size() == t.size() &&
        memcmp(b.tab_uploaded[parity].data(), t.data(), bytes) == 0)
        return true;
    if (fail(b.grids[0], cudaMemcpyAsync(b.dev_tab[parity], t.data(), bytes,
                                         cudaMemcpyHostToDevice, b.stream)))
        return false;
    b.tab_uploaded[parity] = t;
    return true;
}

// The paired launch of every group over device table `parity` (made by
// upload_pair_table with the same groups).
bool build_pair_params(LBMBatch &b, int parity, std::vector<BatchPairParams> &out,
                       std::vector<int> &sets) {
    out.assign(b.groups.size(), BatchPairParams{});
    sets.assign(b.groups.size(), BATCH_SET_ALL);
    size_t base = 0;
    for (size_t gi = 0; gi < b.groups.size(); gi++) {
        const std::vector<int> &grp = b.groups[gi];
        unsigned used = 0;
        long long total = 0;
        for (size_t j = 0; j < grp.size(); j++) {
            const BatchGridDev &e = b.tab[parity][base + j];
            out[gi].starts[j] = (unsigned)total;
            total += (long long)e.tiles_x * e.tiles_y * impl(b.grids[grp[j]])->nz;
            used |= 1u << e.combo;
        }
        if (total > 0x7fffffffLL) return false;
        out[gi].starts[grp.size()] = (unsigned)total;
        out[gi].count = (int)grp.size();
        out[gi].grids = b.dev_tab[parity] + base;
        sets[gi] = set_of(used);
        base += grp.size();
    }
    return true;
}

bool step_fused_pair(LBMBatch &b, const std::vector<BatchPairParams> &p,
                     const std::vector<int> &sets) {
    for (size_t gi = 0; gi < p.size(); gi++)
        if (fail(b.grids[0], launch_step_batch_pair(b.storage, p[gi], sets[gi], b.stream)))
            return false;
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
    b->pair = storage != LBM_STORAGE_FP64;
    for (int i = 0; i < count; i++)
        if (impl(grids[i])->nx % 2 != 0 || impl(grids[i])->n >= (1ll << 31)) b->pair = false;
    b->lbx.assign(count, 5);  // 64 x 4 (pair) or 32 x 8 tiles, the single-grid defaults
    b->grid_done.assign(count, nullptr);
    bool good = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess;
    good = good && cudaEventCreateWithFlags(&b->batch_done, cudaEventDisableTiming) == cudaSuccess;
    good = good && cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess;
    for (int s = 0; good && s < kStreams; s++) {
        good = cudaStreamCreateWithFlags(&b->side[s], cudaStreamNonBlocking) == cudaSuccess;
        good = good &&
               cudaEventCreateWithFlags(&b->side_done[s], cudaEventDisableTiming) == cudaSuccess;
    }
    for (int i = 0; good && i < count; i++)
        good = cudaEventCreateWithFlags(&b->grid_done[i], cudaEventDisableTiming) == cudaSuccess;
    for (int p = 0; good && b->pair && p < 2; p++)
        good = cudaMalloc(&b->dev_tab[p], sizeof(BatchGridDev) * (size_t)count) == cudaSuccess;
    if (!good) {
        LBM_BatchFree(b);
        return nullptr;
    }
    make_groups(*b);
    make_lanes(*b);
    return b;
}

void LBM_BatchFree(LBMBatch *b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(*b);
    for (cudaEvent_t e : b->grid_done)
        if (e) cudaEventDestroy(e);
    if (b->batch_done) cudaEventDestroy(b->batch_done);
    if (b->fork) cudaEventDestroy(b->fork);
    for (int s = 0; s < kStreams; s++) {
        if (b->side[s]) cudaStreamDestroy(b->side[s]);
        if (b->side_done[s]) cudaEventDestroy(b->side_done[s]);
    }
    if (b->stream) cudaStreamDestroy(b->stream);
    for (int p = 0; p < 2; p++)
        if (b->dev_tab[p]) cudaFree(b->dev_tab[p]);
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

    // step arguments of both buffer parities
    make_groups(*b);  // operators may have changed between runs
    for (int p = 0; p < 2; p++) b->args[p].resize(n);
    for (int i = 0; i < n; i++) {
        LBMGrid *g = b->grids[i];
        GridImpl &I = *impl(g);
        if (I.fbuf >= 0 || I.stream_periodic != g->periodicYZ) return LBM_ERR_CUDA;
        b->args[0][i] = step_of(g, I.pop[I.gbuf], I.pop[1 - I.gbuf], inlet + 3 * i);
        b->args[1][i] = step_of(g, I.pop[1 - I.gbuf], I.pop[I.gbuf], inlet + 3 * i);
    }
    if (b->mode == MODE_FUSED && b->pair) {
        if (!upload_pair_table(*b, b->args[0], 0) || !upload_pair_table(*b, b->args[1], 1))
            return LBM_ERR_CUDA;
        if (!build_pair_params(*b, 0, b->pparams[0], b->sets) ||
            !build_pair_params(*b, 1, b->pparams[1], b->sets))
            return LBM_ERR_INVALID_ARGUMENT;
    } else if (b->mode == MODE_FUSED && (!build_params(*b, b->args[0], b->params[0], b->sets) ||
                                         !build_params(*b, b->args[1], b->params[1], b->sets))) {
        return LBM_ERR_INVALID_ARGUMENT;
    }

    // the batch waits for every grid's queued work
    for (int i = 0; i < n; i++) {
        if (fail(b->grids[i], cudaEventRecord(b->grid_done[i], impl(b->grids[i])->stream)))
            return LBM_ERR_CUDA;
        if (fail(b->grids[i], cudaStreamWaitEvent(b->stream, b->grid_done[i], 0)))
            return LBM_ERR_CUDA;
    }
    // `k` steps from parity 0 (k even keeps the parity)
    auto run = [&](int k) {
        if (b->mode == MODE_GRAPH) return k == 0 || steps_graph(*b, b->args, k);
        for (int j = 0; j < k; j++)
            if (!(b->pair ? step_fused_pair(*b, b->pparams[j & 1], b->sets)
                          : step_fused(*b, b->params[j & 1], b->sets)))
                return false;
        return true;
    };
    int left = steps;
    if (left >= kChunk) {
        bool stale = !b->graph || b->graph_mode != b->mode;
        if (!stale && b->mode == MODE_FUSED && b->pair)
            stale = b->graph_sets != b->sets ||
                    !same_pair_params(b->graph_pparams[0], b->pparams[0]) ||
                    !same_pair_params(b->graph_pparams[1], b->pparams[1]);
        else if (!stale && b->mode == MODE_FUSED)
            stale = b->graph_sets != b->sets || !same_params(b->graph_params[0], b->params[0]) ||
                    !same_params(b->graph_params[1], b->params[1]);
        if (!stale && b->mode == MODE_GRAPH)
            stale = b->graph_lbx != b->lbx || !same_arg_vec(b->graph_args[0], b->args[0]) ||
                    !same_arg_vec(b->graph_args[1], b->args[1]);
        if (stale) {
            drop_graph(*b);
            cudaGraph_t graph = nullptr;
            bool good = !fail(g0, cudaStreamBeginCapture(b->stream,
                                                         cudaStreamCaptureModeThreadLocal));
            good = good && run(kChunk);
            const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
            good = good && !fail(g0, e);
            cudaGraphExec_t exec = nullptr;
            if (good) good = !fail(g0, cudaGraphInstantiate(&exec, graph, 0));
            if (graph) cudaGraphDestroy(graph);
            if (!good) return LBM_ERR_CUDA;
            b->graph = exec;
            b->graph_mode = b->mode;
            b->graph_params[0] = b->params[0];
            b->graph_params[1] = b->params[1];
            b->graph_pparams[0] = b->pparams[0];
            b->graph_pparams[1] = b->pparams[1];
            b->graph_sets = b->sets;
            b->graph_args[0] = b->args[0];
            b->graph_args[1] = b->args[1];
            b->graph_lbx = b->lbx;
        }
        while (left >= kChunk) {
            if (fail(g0, cudaGraphLaunch(b->graph, b->stream))) return LBM_ERR_CUDA;
            left -= kChunk;
        }
    }
    if (!run(left)) return LBM_ERR_CUDA;

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
    const int n = b->count;
    // Time the launch each grid's next step would make, in place: once its
    // velocity is materialised, the buffer that step writes holds nothing
    // the grid still needs, and the next step overwrites it anyway.
    unsigned long long *guard = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    bool good = !fail(g0, cudaMalloc(&guard, sizeof(unsigned long long))) &&
                !fail(g0, cudaEventCreate(&t0)) && !fail(g0, cudaEventCreate(&t1));
    std::vector<StepArgs> a(n);
    for (int i = 0; good && i < n; i++) {
        LBMGrid *g = b->grids[i];
        GridImpl &I = *impl(g);
        good = grid_ensure_velocity(g) && !fail(g, cudaStreamSynchronize(I.stream));
        const float in[3] = {I.vin_inlet[0], I.vin_inlet[1], I.vin_inlet[2]};
        a[i] = I.fbuf >= 0 ? step_of(g, I.pop[I.fbuf], I.pop[I.gbuf], in)
                           : step_of(g, I.pop[I.gbuf], I.pop[1 - I.gbuf], in);
        a[i].guard = guard;
    }
    good = good && !fail(g0, cudaStreamSynchronize(b->stream));
    auto timed = [&](auto &&launch) -> float {
        if (!good) return 0.f;
        good = launch();  // one untimed launch first
        good = good && !fail(g0, cudaEventRecord(t0, b->stream));
        for (int k = 0; good && k < trialLaunches; k++) good = launch();
        good = good && !fail(g0, cudaEventRecord(t1, b->stream)) &&
               !fail(g0, cudaEventSynchronize(t1));
        float ms = 0;
        good = good && !fail(g0, cudaEventElapsedTime(&ms, t0, t1));
        return ms;
    };
    // per grid and schedule, the fastest tile shape (a wider tile must be at
    // least 2 % faster to replace a narrower one)
    std::vector<int> lbx_fused(n, 5), lbx_graph(n, 5);
    for (int i = 0; good && i < n; i++) {
        float best_f = 1e30f, best_g = 1e30f;
        for (int l = lbx_min(); good && l <= lbx_max(*b); l++) {
            b->lbx[i] = l;
            float mf = 1e30f;
            if (b->pair) {
                // this grid alone through the paired fused kernel, its entry
                // in device table 0
                const BatchGridDev e = pair_entry(*b, i, a[i]);
                good = !fail(g0, cudaMemcpyAsync(b->dev_tab[0], &e, sizeof(e),
                                                  cudaMemcpyHostToDevice, b->stream)) &&
                       !fail(g0, cudaStreamSynchronize(b->stream));
                BatchPairParams p{};
                p.grids = b->dev_tab[0];
                p.starts[0] = 0;
                p.starts[1] = (unsigned)((long long)e.tiles_x * e.tiles_y * impl(b->grids[i])->nz);
                p.count = 1;
                const int set = set_of(1u << e.combo);
                mf = timed([&] {
                    return !fail(g0, launch_step_batch_pair(b->storage, p, set, b->stream));
                });
            } else {
                BatchLaunchParams p{};
                p.e[0] = make_entry(b->grids[i], l, a[i]);
                p.starts[0] = 0;
                p.starts[1] = (unsigned)units_of(p.e[0], impl(b->grids[i])->nz);
                p.count = 1;
                const int set = set_of(1u << p.e[0].combo);
                mf = timed([&] {
                    return !fail(g0, launch_step_batch(b->storage, p, set, b->stream));
                });
            }
            if (good && mf < best_f * 0.98f) best_f = mf, lbx_fused[i] = l;
            const float mg = timed([&] { return !fail(g0, grid_step(*b, i, a[i], b->stream)); });
            if (good && mg < best_g * 0.98f) best_g = mg, lbx_graph[i] = l;
        }
    }
    // the whole batch, one step, in each schedule with its tiles
    float ms_fused = 1e30f, ms_graph = 1e30f;
    if (good) {
        b->lbx = lbx_fused;
        make_groups(*b);
        std::vector<int> sets;
        if (b->pair) {
            std::vector<BatchPairParams> p;
            b->tab_uploaded[0].clear();  // device table 0 was overwritten above
            good = upload_pair_table(*b, a, 0) && build_pair_params(*b, 0, p, sets);
            ms_fused = timed([&] { return step_fused_pair(*b, p, sets); });
            b->tab_uploaded[0].clear();  // holds the trial arguments now
        } else {
            std::vector<BatchLaunchParams> p;
            good = build_params(*b, a, p, sets);
            ms_fused = timed([&] { return step_fused(*b, p, sets); });
        }
    }
    if (good) {
        b->lbx = lbx_graph;
        const std::vector<StepArgs> both[2] = {a, a};
        ms_graph = timed([&] { return steps_graph(*b, both, 1); });
    }
    if (good) {
        b->mode = ms_graph < ms_fused ? MODE_GRAPH : MODE_FUSED;
        b->lbx = b->mode == MODE_GRAPH ? lbx_graph : lbx_fused;
        drop_graph(*b);
    }
    good = good && !fail(g0, cudaStreamSynchronize(b->stream));
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(guard);
    return good ? LBM_OK : LBM_ERR_CUDA;
}

int LBM_BatchGetTile(LBMBatch *b, int index, int *tileX, int *tileY) {
    if (!b || index < 0 || index >= b->count || !tileX || !tileY) return LBM_ERR_INVALID_ARGUMENT;
    *tileX = tile_x_cells(*b, b->lbx[index]);
    *tileY = tile_y_cells(*b, b->lbx[index]);
    return LBM_OK;
}

int LBM_BatchSetTile(LBMBatch *b, int index, int tileX) {
    if (!b || index < 0 || index >= b->count) return LBM_ERR_INVALID_ARGUMENT;
    int lbx = -1;
    for (int k = lbx_min(); k <= lbx_max(*b); k++)
        if (tileX == tile_x_cells(*b, k)) lbx = k;
    if (lbx < 0) return LBM_ERR_INVALID_ARGUMENT;
    if (b->lbx[index] != lbx) drop_graph(*b);
    b->lbx[index] = lbx;
    return LBM_OK;
}

int LBM_BatchGetSchedule(LBMBatch *b) { return b ? b->mode : -1; }

int LBM_BatchSetSchedule(LBMBatch *b, int schedule) {
    if (!b || (schedule != MODE_FUSED && schedule != MODE_GRAPH)) return LBM_ERR_INVALID_ARGUMENT;
    if (b->mode != schedule) drop_graph(*b);
    b->mode = schedule;
    return LBM_OK;
}

long long LBM_BatchTilesPerStep(LBMBatch *b) {
    if (!b) return 0;
    long long total = 0;
    for (int i = 0; i < b->count; i++) {
        const int bx = tile_x_cells(*b, b->lbx[i]), by = tile_y_cells(*b, b->lbx[i]);
        const GridImpl &I = *impl(b->grids[i]);
        total += (long long)((I.nx + bx - 1) / bx) * ((I.ny + by - 1) / by) * I.nz;
    }
    return total;
}

void *LBM_BatchGetStream(LBMBatch *b) { return b ? (void *)b->stream : nullptr; }

}  // extern "C"
