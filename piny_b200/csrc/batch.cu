// Many boxes per step, and the launch-shape autotuner.
//
// A batch holds the contexts of independent boxes (different sizes, bead
// counts and meshes).  One call enqueues every box's whole evaluation --
// positions in, list-based pair forces, PME, intramolecular terms, forces
// out, energy sums to pinned host memory -- in one of two forms:
//   multi-box kernels: each phase is one persistent launch per group of
//     boxes that share its compile-time shape (boxtab.cuh); the groups'
//     PME chains, pair launches and the intramolecular launch are parallel
//     graph branches between the staging and the finishing launches -- a
//     few dozen launches for any number of boxes;
//   branches: every box's own kernels as a parallel branch forked from and
//     joined to one stream (for boxes the multi-box kernels do not cover).
// The first call (and any call whose device pointers, cells or flags differ
// from the previous one) captures that work into a CUDA graph; every call
// launches the graph once and then does the host bookkeeping of each box.
//
// The autotuner times, on the caller's own inputs, the launch shapes a
// context can run with -- PME tile edge (8 or 16 grid points), pair kernel
// (molecule-pair or site-list), pair grid size (blocks per SM) and PME
// overlap with the pair kernel -- keeps the fastest, and remembers it per
// system shape for the rest of the process.
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "common.cuh"

using namespace pinyb200;

namespace {

// process-wide tuning results per system shape
typedef std::tuple<int, int, int, int, int, int, int, int> TuneKey;
std::mutex g_tune_mu;
std::map<TuneKey, std::vector<int>> g_tune;

TuneKey tune_key(const pinyb200_ctx *c)
{
    return TuneKey(c->sys.natm, c->P, c->sys.ngrid[0], c->sys.ngrid[1], c->sys.ngrid[2], c->sys.n_interp,
                   c->precision, (int)(c->use_mol && c->mol_ok));
}

void get_choice(const pinyb200_ctx *c, int *ch)
{
    ch[0] = c->pme_tile;
    ch[1] = c->pair_variant;
    ch[2] = c->pair_blocks_per_sm;
    ch[3] = c->pme_overlap ? 1 : 0;
}

int set_choice(pinyb200_ctx *c, const int *ch)
{
    if (!(ch[0] == 8 || ch[0] == 16) || !(ch[1] >= 0 && ch[1] <= 2) || ch[2] < 1 || ch[2] > 64 ||
        !(ch[3] == 0 || ch[3] == 1))
        return record_error(c, PINYB200_ERR_ARG,
                            "tuning: expected {tile 8|16, pair 0|1|2, blocks/SM 1..64, overlap 0|1}");
    if (c->sys.nchrg > 0 && c->sys.nktot > 0 && ch[0] != c->pme_tile) {
        int rc = pme_tiles_resize(c, ch[0]);
        if (rc) return rc;
    }
    c->pair_variant = ch[1];
    c->pair_blocks_per_sm = ch[2];
    c->pme_overlap = ch[3] != 0;
    c->gen++;
    return PINYB200_OK;
}

}  // namespace

struct pinyb200_batch {
    int device = 0;
    std::vector<pinyb200_ctx *> box;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    double *h_acc = nullptr;         // pinned, per box [P][S_NSLOT]
    std::vector<size_t> acc_off;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // what the captured graph was built for
    std::vector<const void *> key_ptr;
    std::vector<double> key_h;
    int key_flags = -1;
    float last_ms = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    // the multi-box form: one graph branch per shape group (streams reused
    // round-robin past the pool), a join event per branch
    std::vector<cudaStream_t> gstream;
    std::vector<cudaEvent_t> gjoin;
    cudaEvent_t pfork = nullptr;
    int fused = 0;     // form of the captured graph
    int launches = 0;  // kernel nodes of the captured graph
    std::string err;
};

namespace {

int bfail(pinyb200_batch *bt, int code, const std::string &msg)
{
    if (bt) bt->err = msg;
    return record_error(nullptr, code, msg);
}

#define BCK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return bfail(bt, PINYB200_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

// Whether the multi-box kernels cover every box of the call: MIXED
// molecule-pair kernel with a known site pattern, orthorhombic cells,
// compact PME records, flags they serve.
bool fused_ok(const pinyb200_batch *bt, const double *const *hmat, int flags)
{
    if (flags & (PINYB200_UPDATE_LIST | PINYB200_SITE_PAIRS | PINYB200_BATCH_BRANCHES)) return false;
    for (size_t i = 0; i < bt->box.size(); i++) {
        const pinyb200_ctx *c = bt->box[i];
        const double *h = hmat[i];
        const bool ortho = h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0 && h[5] == 0.0 && h[6] == 0.0 && h[7] == 0.0;
        if (c->precision != PINYB200_MIXED || !c->use_mol || !c->mol_ok || !c->mix_ok || mix_pattern(c) == 0 ||
            !ortho || c->pme_full_records || c->sm_count != bt->box[0]->sm_count)
            return false;
    }
    return true;
}

// Every box's evaluation as multi-box kernels on bt->stream: the work of
// enqueue_device for each box, phase by phase.
int fused_enqueue(pinyb200_batch *bt, const double *const *d_pos, const double *const *d_xmod,
                  const double *const *hmat, int flags, double *const *d_force)
{
    const int nbox = (int)bt->box.size();
    const int sm = bt->box[0]->sm_count;
    const bool energy = !(flags & PINYB200_NO_ENERGY);
    cudaStream_t st = bt->stream;
    std::vector<Cell> cells;
    std::vector<const double *> pos;
    std::vector<double *> force;
    std::vector<std::pair<void *, size_t>> zero;
    std::vector<CopySeg> xm, acc;
    for (int i = 0; i < nbox; i++) {
        pinyb200_ctx *c = bt->box[i];
        cells.push_back(cell_from_hmat(hmat[i]));
        pos.push_back(d_pos[i]);
        force.push_back(d_force[i]);
        const size_t nb = (size_t)c->sys.natm * 3 * c->P;
        zero.emplace_back(c->d_forceT, nb * sizeof(double));
        zero.emplace_back(c->d_acc, (size_t)c->P * S_NSLOT * sizeof(double));
        if (c->P > 1) {
            const double *src = d_xmod ? d_xmod[i] : nullptr;
            if (src != c->d_xmod) xm.push_back(CopySeg{src, c->d_posT, c->d_xmod, (long long)c->sys.natm * 3, c->P});
        }
        if (energy)
            acc.push_back(CopySeg{c->d_acc, nullptr, bt->h_acc + bt->acc_off[i], (long long)c->P * S_NSLOT, 1});
    }
    cudaError_t e = launch_zero_batch(zero, sm, st);
    if (e == cudaSuccess) e = launch_transpose_in_batch(bt->box, pos, sm, st);
    if (e == cudaSuccess && !xm.empty()) e = launch_copy_batch(xm, sm, st);
    if (e == cudaSuccess) e = launch_ghost_batch(bt->box, false, sm, st);
    if (e == cudaSuccess) e = launch_mol_extent_batch(bt->box, sm, st);
    // The force terms as parallel branches: one per PME shape group (order,
    // tile edge, mesh: its whole chain of launches), one per pair-kernel
    // group (bead count, site pattern), one for the intramolecular terms;
    // heaviest first.  Independent groups overlap, so no launch's tail
    // leaves the GPU idle while other groups still have work.
    struct Branch {
        int kind;  // 0 PME, 1 pair, 2 intramolecular
        std::vector<pinyb200_ctx *> box;
        std::vector<Cell> cell;
        double work;
    };
    std::map<std::tuple<int, int, int, int, int, int>, Branch> groups;
    for (int i = 0; i < nbox; i++) {
        pinyb200_ctx *c = bt->box[i];
        const double G = (double)c->sys.ngrid[0] * c->sys.ngrid[1] * c->sys.ngrid[2];
        if (c->sys.nchrg > 0 && c->sys.nktot > 0) {
            Branch &b = groups[std::make_tuple(0, c->sys.n_interp, c->pme_tile, c->sys.ngrid[0], c->sys.ngrid[1],
                                               c->sys.ngrid[2])];
            b.kind = 0;
            b.box.push_back(c);
            b.cell.push_back(cells[i]);
            b.work += (G + 40.0 * c->sys.nchrg) * c->P;
        }
        Branch &q = groups[std::make_tuple(1, c->P, mix_pattern(c), 0, 0, 0)];
        q.kind = 1;
        q.box.push_back(c);
        q.cell.push_back(cells[i]);
        q.work += 300.0 * c->chunk_cap * c->P;
    }
    std::vector<Branch> br;
    for (auto &kv : groups) br.push_back(kv.second);
    br.push_back(Branch{2, bt->box, cells, 0.0});
    std::stable_sort(br.begin(), br.end(), [](const Branch &x, const Branch &y) { return x.work > y.work; });
    const size_t npool = 12;
    while (e == cudaSuccess && bt->gstream.size() < std::min(npool, br.size())) {
        cudaStream_t s = nullptr;
        e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e == cudaSuccess) bt->gstream.push_back(s);
    }
    while (e == cudaSuccess && bt->gjoin.size() < br.size()) {
        cudaEvent_t ev = nullptr;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) bt->gjoin.push_back(ev);
    }
    if (e == cudaSuccess) e = cudaEventRecord(bt->pfork, st);
    for (size_t k = 0; k < br.size() && e == cudaSuccess; k++) {
        cudaStream_t s = bt->gstream[k % bt->gstream.size()];
        e = cudaStreamWaitEvent(s, bt->pfork, 0);
        if (e != cudaSuccess) break;
        if (br[k].kind == 0) e = launch_pme_batch(br[k].box, br[k].cell, energy, sm, s);
        else if (br[k].kind == 1) e = launch_mol_pair_mixed_batch(br[k].box, br[k].cell, energy, sm, s);
        else e = launch_intra_batch(br[k].box, energy, sm, s);
        if (e == cudaSuccess) e = cudaEventRecord(bt->gjoin[k], s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, bt->gjoin[k], 0);
    }
    if (e == cudaSuccess) e = launch_pme_force_add_batch(bt->box, sm, st);
    if (e == cudaSuccess && (flags & PINYB200_DISTRIB_GHOSTS)) e = launch_ghost_batch(bt->box, true, sm, st);
    if (e == cudaSuccess) e = launch_transpose_out_batch(bt->box, force, sm, st);
    // per-bead sums straight into the pinned host buffer
    if (e == cudaSuccess && energy) e = launch_copy_batch(acc, sm, st);
    if (e != cudaSuccess) return bfail(bt, PINYB200_ERR_CUDA, std::string("batch kernels: ") + cudaGetErrorString(e));
    return PINYB200_OK;
}

int count_kernel_nodes(cudaGraph_t g)
{
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return 0;
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
    int k = 0;
    for (size_t i = 0; i < n; i++) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
    }
    return k;
}

void drop_graph(pinyb200_batch *bt)
{
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    bt->exec = nullptr;
    bt->graph = nullptr;
}

// Capture one form of the batch call into a graph: the multi-box kernels
// (after one plain run of them, so that kernel attributes and occupancy
// queries happen outside the capture) or one branch per box.
int capture_form(pinyb200_batch *bt, bool fused, const double *const *d_pos, const double *const *d_xmod,
                 const double *const *hmat, int flags, double *const *d_force, cudaGraph_t *out,
                 cudaGraphExec_t *exec)
{
    const int nbox = (int)bt->box.size();
    *out = nullptr;
    *exec = nullptr;
    if (fused) {
        int rc = fused_enqueue(bt, d_pos, d_xmod, hmat, flags, d_force);
        if (rc) return rc;
        BCK(cudaStreamSynchronize(bt->stream));
    }
    BCK(cudaStreamBeginCapture(bt->stream, cudaStreamCaptureModeRelaxed));
    int rc = PINYB200_OK;
    cudaError_t ce = fused ? cudaSuccess : cudaEventRecord(bt->fork, bt->stream);
    if (fused) rc = fused_enqueue(bt, d_pos, d_xmod, hmat, flags, d_force);
    for (int i = 0; i < nbox && !fused && ce == cudaSuccess && rc == PINYB200_OK; i++) {
        pinyb200_ctx *c = bt->box[i];
        ce = cudaStreamWaitEvent(c->stream, bt->fork, 0);
        if (ce != cudaSuccess) break;
        const Cell cell = cell_from_hmat(hmat[i]);
        rc = enqueue_device(c, d_pos[i], d_xmod ? d_xmod[i] : nullptr, cell, flags, d_force[i], false,
                            bt->h_acc + bt->acc_off[i]);
        if (rc) break;
        ce = cudaEventRecord(bt->join[i], c->stream);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(bt->stream, bt->join[i], 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(bt->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return fused ? rc : bfail(bt, rc, "batch capture: enqueue failed");
    }
    if (ce != cudaSuccess || ee != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return bfail(bt, PINYB200_ERR_CUDA,
                     std::string("batch capture: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ee));
    }
    const cudaError_t ei = cudaGraphInstantiate(exec, g, 0);
    if (ei != cudaSuccess) {
        cudaGraphDestroy(g);
        *exec = nullptr;
        return bfail(bt, PINYB200_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(ei));
    }
    *out = g;
    return PINYB200_OK;
}

}  // namespace

extern "C" {

int pinyb200_get_tuning(pinyb200_ctx *c, int *choice)
{
    if (!c || !choice) return record_error(c, PINYB200_ERR_ARG, "get_tuning: NULL");
    get_choice(c, choice);
    return PINYB200_OK;
}

int pinyb200_set_tuning(pinyb200_ctx *c, const int *choice)
{
    if (!c || !choice) return record_error(c, PINYB200_ERR_ARG, "set_tuning: NULL");
    if (cudaSetDevice(c->device) != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, "set_tuning: device");
    return set_choice(c, choice);
}

int pinyb200_autotune(pinyb200_ctx *c, const double *d_pos, const double *d_xmod, const double *hmat, int flags,
                      int reps, int *choice, float *best_ms)
{
    if (!c || !d_pos || !hmat) return record_error(c, PINYB200_ERR_ARG, "autotune: NULL argument");
    if (!c->have_list) return record_error(c, PINYB200_ERR_STATE, "autotune: build the Verlet list first");
    if (cudaSetDevice(c->device) != cudaSuccess) return record_error(c, PINYB200_ERR_CUDA, "autotune: device");
    if (reps < 1) reps = 3;
    const TuneKey key = tune_key(c);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end() && !(flags & PINYB200_TUNE_AGAIN)) {
            int rc = set_choice(c, it->second.data());
            if (rc) return rc;
            if (choice) get_choice(c, choice);
            if (best_ms) *best_ms = -1.0f;
            return PINYB200_OK;
        }
    }
    const int eflags = flags & ~PINYB200_TUNE_AGAIN;
    const Cell cell = cell_from_hmat(hmat);
    const bool has_pme = c->sys.nchrg > 0 && c->sys.nktot > 0;
    const int nmin = std::min(c->sys.ngrid[0], std::min(c->sys.ngrid[1], c->sys.ngrid[2]));
    std::vector<int> tiles = {8};
    if (has_pme && nmin >= 16) tiles.push_back(16);
    std::vector<int> variants = {1};
    if (c->use_mol && c->mol_ok) variants.insert(variants.begin(), 0);
    if (c->use_mol && c->mol_ok && c->mix_ok) variants.push_back(2);
    const int bps[5] = {4, 5, 8, 16, 32};
    int best[4];
    get_choice(c, best);
    float tbest = 1e30f;
    for (int T : tiles)
        for (int v : variants)
            for (int bp : bps)
                for (int ov = 0; ov < 2; ov++) {
                    const int ch[4] = {has_pme ? T : c->pme_tile, v, bp, ov};
                    int rc = set_choice(c, ch);
                    if (rc) return rc;
                    float tsum = 0;
                    for (int r = 0; r <= reps; r++) {
                        rc = enqueue_device(c, d_pos, d_xmod, cell, eflags, c->d_force_aos, true, nullptr);
                        if (rc) return rc;
                        if (cudaStreamSynchronize(c->stream) != cudaSuccess)
                            return record_error(c, PINYB200_ERR_CUDA, "autotune: synchronize");
                        float ms = 0;
                        cudaEventElapsedTime(&ms, c->ev[0], c->ev[4]);
                        if (r > 0) tsum += ms;  // the first run of each shape warms up
                    }
                    const float t = tsum / reps;
                    if (t < tbest) {
                        tbest = t;
                        for (int k = 0; k < 4; k++) best[k] = ch[k];
                    }
                    if (!has_pme) break;  // overlap has nothing to overlap
                }
    int rc = set_choice(c, best);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune[key] = std::vector<int>(best, best + 4);
    }
    if (choice) get_choice(c, choice);
    if (best_ms) *best_ms = tbest;
    return PINYB200_OK;
}

int pinyb200_batch_create(pinyb200_ctx *const *ctx, int nbox, pinyb200_batch **out)
{
    if (!ctx || nbox < 1 || !out) return record_error(nullptr, PINYB200_ERR_ARG, "batch_create: bad arguments");
    for (int i = 0; i < nbox; i++) {
        if (!ctx[i]) return record_error(nullptr, PINYB200_ERR_ARG, "batch_create: NULL context");
        if (ctx[i]->device != ctx[0]->device)
            return record_error(nullptr, PINYB200_ERR_ARG, "batch_create: contexts on different devices");
        for (int j = 0; j < i; j++)
            if (ctx[j] == ctx[i]) return record_error(nullptr, PINYB200_ERR_ARG, "batch_create: context listed twice");
    }
    pinyb200_batch *bt = new pinyb200_batch();
    bt->device = ctx[0]->device;
    bt->box.assign(ctx, ctx + nbox);
    *out = nullptr;
    auto cleanup = [&](int rc) {
        pinyb200_batch_destroy(bt);
        return rc;
    };
    if (cudaSetDevice(bt->device) != cudaSuccess) return cleanup(bfail(nullptr, PINYB200_ERR_CUDA, "batch: device"));
    if (cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&bt->pfork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&bt->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&bt->ev[0]) != cudaSuccess || cudaEventCreate(&bt->ev[1]) != cudaSuccess)
        return cleanup(bfail(nullptr, PINYB200_ERR_CUDA, "batch: stream/event creation failed"));
    bt->join.assign(nbox, nullptr);
    size_t nacc = 0;
    for (int i = 0; i < nbox; i++) {
        if (cudaEventCreateWithFlags(&bt->join[i], cudaEventDisableTiming) != cudaSuccess)
            return cleanup(bfail(nullptr, PINYB200_ERR_CUDA, "batch: event creation failed"));
        bt->acc_off.push_back(nacc);
        nacc += (size_t)ctx[i]->P * S_NSLOT;
    }
    if (cudaMallocHost(&bt->h_acc, nacc * sizeof(double)) != cudaSuccess)
        return cleanup(bfail(nullptr, PINYB200_ERR_CUDA, "batch: pinned buffer"));
    *out = bt;
    return PINYB200_OK;
}

int pinyb200_batch_destroy(pinyb200_batch *bt)
{
    if (!bt) return PINYB200_OK;
    cudaSetDevice(bt->device);
    drop_graph(bt);
    for (cudaEvent_t e : bt->join)
        if (e) cudaEventDestroy(e);
    if (bt->fork) cudaEventDestroy(bt->fork);
    if (bt->pfork) cudaEventDestroy(bt->pfork);
    for (cudaEvent_t e : bt->gjoin) cudaEventDestroy(e);
    for (cudaStream_t s : bt->gstream) cudaStreamDestroy(s);
    for (int i = 0; i < 2; i++)
        if (bt->ev[i]) cudaEventDestroy(bt->ev[i]);
    if (bt->stream) cudaStreamDestroy(bt->stream);
    if (bt->h_acc) cudaFreeHost(bt->h_acc);
    delete bt;
    return PINYB200_OK;
}

int pinyb200_batch_energy_force_device(pinyb200_batch *bt, const double *const *d_pos, const double *const *d_xmod,
                                       const double *const *hmat, int flags, double *const *d_force,
                                       pinyb200_energies *e, void *stream)
{
    if (!bt || !d_pos || !hmat || !d_force) return bfail(bt, PINYB200_ERR_ARG, "batch_energy_force: NULL argument");
    const int nbox = (int)bt->box.size();
    for (int i = 0; i < nbox; i++) {
        if (!d_pos[i] || !hmat[i] || !d_force[i]) return bfail(bt, PINYB200_ERR_ARG, "batch_energy_force: NULL box input");
        if (!bt->box[i]->have_list) return bfail(bt, PINYB200_ERR_STATE, "batch_energy_force: a box has no list");
    }
    BCK(cudaSetDevice(bt->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : bt->stream;
    // does the captured graph still describe this call?
    std::vector<const void *> kp;
    std::vector<double> kh;
    for (int i = 0; i < nbox; i++) {
        kp.push_back(d_pos[i]);
        kp.push_back(d_xmod ? d_xmod[i] : nullptr);
        kp.push_back(d_force[i]);
        kh.insert(kh.end(), hmat[i], hmat[i] + 9);
        kh.push_back((double)bt->box[i]->gen);  // a list build or retune invalidates the graph
    }
    if (!bt->exec || kp != bt->key_ptr || kh != bt->key_h || flags != bt->key_flags) {
        drop_graph(bt);
        // one plain run per box first: builds the influence functions for
        // these cells and sets kernel attributes outside the capture
        for (int i = 0; i < nbox; i++) {
            pinyb200_ctx *c = bt->box[i];
            const Cell cell = cell_from_hmat(hmat[i]);
            int rc = enqueue_device(c, d_pos[i], d_xmod ? d_xmod[i] : nullptr, cell, flags, d_force[i], false, nullptr);
            if (rc) return bfail(bt, rc, std::string("batch warm-up: ") + pinyb200_last_error(c));
            BCK(cudaStreamSynchronize(c->stream));
        }
        // the forms to capture: the multi-box kernels where they cover the
        // boxes, the branches otherwise; both, when neither is asked for,
        // and the faster one is kept (timed on these inputs)
        const bool can_fuse = fused_ok(bt, hmat, flags);
        std::vector<int> forms;
        if (!can_fuse) forms = {0};
        else if (flags & PINYB200_BATCH_KERNELS) forms = {1};
        else forms = {1, 0};
        float tbest = 1e30f;
        for (int form : forms) {
            cudaGraph_t g = nullptr;
            cudaGraphExec_t x = nullptr;
            int rc = capture_form(bt, form == 1, d_pos, d_xmod, hmat, flags, d_force, &g, &x);
            if (rc) {
                drop_graph(bt);
                return rc;
            }
            float t = 0.0f;
            if (forms.size() > 1) {
                for (int r = 0; r < 2; r++) {
                    BCK(cudaEventRecord(bt->ev[0], bt->stream));
                    BCK(cudaGraphLaunch(x, bt->stream));
                    BCK(cudaEventRecord(bt->ev[1], bt->stream));
                    BCK(cudaStreamSynchronize(bt->stream));
                    BCK(cudaEventElapsedTime(&t, bt->ev[0], bt->ev[1]));
                }
            }
            if (t < tbest) {
                drop_graph(bt);
                tbest = t;
                bt->graph = g;
                bt->exec = x;
                bt->fused = form;
                bt->launches = count_kernel_nodes(g);
            } else {
                cudaGraphExecDestroy(x);
                cudaGraphDestroy(g);
            }
        }
        bt->key_ptr = kp;
        bt->key_h = kh;
        bt->key_flags = flags;
    }
    BCK(cudaEventRecord(bt->ev[0], st));
    BCK(cudaGraphLaunch(bt->exec, st));
    BCK(cudaEventRecord(bt->ev[1], st));
    BCK(cudaStreamSynchronize(st));
    BCK(cudaEventElapsedTime(&bt->last_ms, bt->ev[0], bt->ev[1]));
    if (e) {
        const bool energy = !(flags & PINYB200_NO_ENERGY);
        for (int i = 0; i < nbox; i++)
            evaluate_finish(bt->box[i], cell_from_hmat(hmat[i]), flags, energy ? bt->h_acc + bt->acc_off[i] : nullptr,
                            &e[i]);
    }
    return PINYB200_OK;
}

int pinyb200_batch_last_ms(pinyb200_batch *bt, float *ms)
{
    if (!bt || !ms) return bfail(bt, PINYB200_ERR_ARG, "batch_last_ms: NULL");
    *ms = bt->last_ms;
    return PINYB200_OK;
}

int pinyb200_batch_last_mode(pinyb200_batch *bt, int *fused, int *launches)
{
    if (!bt) return bfail(bt, PINYB200_ERR_ARG, "batch_last_mode: NULL");
    if (fused) *fused = bt->fused;
    if (launches) *launches = bt->launches;
    return PINYB200_OK;
}

const char *pinyb200_batch_last_error(pinyb200_batch *bt) { return bt ? bt->err.c_str() : ""; }

}  // extern "C"
