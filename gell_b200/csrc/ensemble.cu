// ensemble.cu — many independent simulations (contexts) stepped together.
//
// Each member is an ordinary context with its own grid, cells and substrates.  The ensemble
// captures two mechanics steps of every member into ONE CUDA graph: an origin stream forks into
// `branches` streams, member i runs on branch i mod branches, and the branches join back, so the
// small kernels of different members run side by side and fill the GPU that any one of them would
// leave mostly idle.  The graph is replayed for every pair of steps and captured again when a
// member's cell count, substrates or double-buffer assignment, or the substep count, changed.
// gell_ensemble_tune times a few branch counts and sweep tile widths and keeps the fastest.
//
// Batched (gell_ensemble_set_batched, or chosen by the tuner): each captured step is the FM_update
// and PreLOD of ALL members as one launch per kernel (gell::mech_batch_step: keys, the sort's
// passes, gather, force and move, the uptake map), then their LOD substeps as one launch per sweep
// axis (and one for the uptake source) over a device-side work list of every member's line tiles
// (gell::lod_batch_run), instead of per-member launches on the branches.  Ensembles beyond the
// batched mechanics' limits (64 members, 4 substrates each) run their mechanics on the branches.
#include <initializer_list>
#include <vector>

#include "gell_internal.cuh"

struct gell_ensemble {
    std::vector<gell_ctx*> m;
    cudaStream_t origin = nullptr;
    std::vector<cudaStream_t> pool;
    cudaEvent_t fork = nullptr, done = nullptr;
    std::vector<cudaEvent_t> join, ready;
    int branches = 0;     // branch streams in use
    int sweep_warps = 0;  // GELL_OPT_SWEEP_WARPS given to every member (0 = each member's default)
    bool batched = false;  // LOD substeps of all members as one launch per sweep (gell::lod_batch_run)
    gell::LodBatch* batch = nullptr;
    cudaGraphExec_t exec = nullptr;
    // what the graph was captured for
    int key_substeps = -1, key_branches = -1, key_warps = -1, key_batched = -1;
    std::vector<int> key_n, key_nsub;
    std::vector<uint32_t> key_par;
    std::vector<long long> launches;  // kernels per member in one replay
};

namespace {

constexpr int kMaxBranches = 64;

bool key_matches(const gell_ensemble* e, int substeps) {
    if (!e->exec || e->key_substeps != substeps || e->key_branches != e->branches || e->key_warps != e->sweep_warps ||
        e->key_batched != (int)e->batched)
        return false;
    for (size_t i = 0; i < e->m.size(); ++i) {
        const gell_ctx* c = e->m[i];
        if (e->key_n[i] != c->n || e->key_nsub[i] != (int)c->subs.size() || e->key_par[i] != gell::buffer_parity(c))
            return false;
    }
    return true;
}

// Capture two mechanics steps of every member into e->exec.
gell_status capture(gell_ensemble* e, int substeps) {
    if (e->exec) {
        cudaGraphExecDestroy(e->exec);
        e->exec = nullptr;
    }
    const size_t n = e->m.size();
    const int nb = e->branches;
    std::vector<cudaStream_t> saved(n);
    std::vector<long long> l0(n);
    for (size_t i = 0; i < n; ++i) {
        saved[i] = e->m[i]->stream;
        l0[i] = e->m[i]->launches;
    }
    if (e->batched) {
        // the work list of every member's substrates, built outside the capture
        gell::lod_batch_free(e->batch);
        e->batch = nullptr;
        if (gell_status bs = gell::lod_batch_build(e->m, &e->batch)) return bs;
    }
    if (cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return GELL_ERR_CUDA;
    gell_status st = GELL_OK;
    cudaError_t ce = cudaSuccess;
    // batched: per step, every member's mechanics (FM_update, PreLOD) on the branches, joined, then
    // all members' LOD substeps as one launch per sweep on the origin stream; otherwise each member's
    // two whole steps on its branch
    const int rounds = e->batched ? 2 : 1;
    // batched: every member's FM_update and PreLOD as one launch per kernel too, when they fit
    const bool mech_batched = e->batched && gell::mech_batch_ok(e->m);
    for (int r = 0; r < rounds && ce == cudaSuccess && st == GELL_OK; ++r) {
        if (mech_batched) {
            st = gell::mech_batch_step(e->m, e->origin);
            if (st == GELL_OK) st = gell::lod_batch_run(e->batch, e->origin, substeps);
            continue;
        }
        ce = cudaEventRecord(e->fork, e->origin);
        for (int b = 0; b < nb && ce == cudaSuccess; ++b) ce = cudaStreamWaitEvent(e->pool[b], e->fork, 0);
        for (size_t i = 0; i < n && ce == cudaSuccess && st == GELL_OK; ++i) {
            gell_ctx* c = e->m[i];
            c->stream = e->pool[i % nb];
            st = gell::one_mechanics_step(c, e->batched ? 0 : substeps);
            if (st == GELL_OK && !e->batched) st = gell::one_mechanics_step(c, substeps);
        }
        for (int b = 0; b < nb && ce == cudaSuccess; ++b) {
            ce = cudaEventRecord(e->join[b], e->pool[b]);
            if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->origin, e->join[b], 0);
        }
        if (e->batched && ce == cudaSuccess && st == GELL_OK) st = gell::lod_batch_run(e->batch, e->origin, substeps);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(e->origin, &g);
    for (size_t i = 0; i < n; ++i) {
        gell_ctx* c = e->m[i];
        c->stream = saved[i];
        e->launches[i] = c->launches - l0[i];  // counted when the graph is replayed
        c->launches = l0[i];
    }
    if (st != GELL_OK || ce != cudaSuccess || ee != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return st != GELL_OK ? st : GELL_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(&e->exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        e->exec = nullptr;
        cudaGetLastError();
        return GELL_ERR_CUDA;
    }
    e->key_substeps = substeps;
    e->key_branches = nb;
    e->key_warps = e->sweep_warps;
    e->key_batched = (int)e->batched;
    for (size_t i = 0; i < n; ++i) {
        e->key_n[i] = e->m[i]->n;
        e->key_nsub[i] = (int)e->m[i]->subs.size();
        e->key_par[i] = gell::buffer_parity(e->m[i]);
    }
    return GELL_OK;
}

// The origin stream waits for every member's queued work (and its queued transfers).
gell_status gather(gell_ensemble* e) {
    for (size_t i = 0; i < e->m.size(); ++i) {
        gell_ctx* c = e->m[i];
        if (gell_status st = gell::cells_begin(c)) return st;
        if (cudaEventRecord(e->ready[i], c->stream) != cudaSuccess ||
            cudaStreamWaitEvent(e->origin, e->ready[i], 0) != cudaSuccess)
            return GELL_ERR_CUDA;
    }
    return GELL_OK;
}

// Every member's stream waits for the work queued on the origin stream.
gell_status scatter(gell_ensemble* e) {
    if (cudaEventRecord(e->done, e->origin) != cudaSuccess) return GELL_ERR_CUDA;
    for (gell_ctx* c : e->m)
        if (cudaStreamWaitEvent(c->stream, e->done, 0) != cudaSuccess) return GELL_ERR_CUDA;
    return GELL_OK;
}

void apply_warps(gell_ensemble* e) {
    for (gell_ctx* c : e->m) c->sweep_warps = e->sweep_warps;
}

}  // namespace

extern "C" {

gell_status gell_ensemble_create(gell_ctx* const* members, int count, gell_ensemble** out) {
    if (!members || count < 1 || !out) return GELL_ERR_INVALID_ARG;
    *out = nullptr;
    for (int i = 0; i < count; ++i) {
        if (!members[i]) return GELL_ERR_INVALID_ARG;
        for (int j = 0; j < i; ++j)
            if (members[j] == members[i]) return GELL_ERR_INVALID_ARG;  // each context once
    }
    gell_ensemble* e = new gell_ensemble;
    e->m.assign(members, members + count);
    const int nb = count < kMaxBranches ? count : kMaxBranches;
    bool ok = cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming) == cudaSuccess;
    e->pool.assign(nb, nullptr);
    e->join.assign(nb, nullptr);
    for (int b = 0; ok && b < nb; ++b)
        ok = cudaStreamCreateWithFlags(&e->pool[b], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&e->join[b], cudaEventDisableTiming) == cudaSuccess;
    e->ready.assign(count, nullptr);
    for (int i = 0; ok && i < count; ++i) ok = cudaEventCreateWithFlags(&e->ready[i], cudaEventDisableTiming) == cudaSuccess;
    e->key_n.assign(count, -1);
    e->key_nsub.assign(count, -1);
    e->key_par.assign(count, 0);
    e->launches.assign(count, 0);
    e->branches = nb;
    if (!ok) {
        cudaGetLastError();
        gell_ensemble_destroy(e);
        return GELL_ERR_CUDA;
    }
    *out = e;
    return GELL_OK;
}

gell_status gell_ensemble_destroy(gell_ensemble* e) {
    if (!e) return GELL_ERR_INVALID_ARG;
    if (e->origin) cudaStreamSynchronize(e->origin);
    if (e->exec) cudaGraphExecDestroy(e->exec);
    for (auto s : e->pool)
        if (s) cudaStreamDestroy(s);
    for (auto v : e->join)
        if (v) cudaEventDestroy(v);
    for (auto v : e->ready)
        if (v) cudaEventDestroy(v);
    gell::lod_batch_free(e->batch);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->done) cudaEventDestroy(e->done);
    if (e->origin) cudaStreamDestroy(e->origin);
    delete e;
    return GELL_OK;
}

gell_status gell_ensemble_configure(gell_ensemble* e, int branches, int sweep_warps) {
    if (!e || branches < 1 || sweep_warps < 0 || sweep_warps > 4) return GELL_ERR_INVALID_ARG;
    const int nb = (int)e->pool.size();
    e->branches = branches < nb ? branches : nb;
    e->sweep_warps = sweep_warps;
    apply_warps(e);
    return GELL_OK;
}

gell_status gell_ensemble_set_batched(gell_ensemble* e, int on) {
    if (!e) return GELL_ERR_INVALID_ARG;
    e->batched = on != 0;
    return GELL_OK;
}

gell_status gell_ensemble_get_batched(const gell_ensemble* e, int* on) {
    if (!e || !on) return GELL_ERR_INVALID_ARG;
    *on = e->batched ? 1 : 0;
    return GELL_OK;
}

gell_status gell_ensemble_run_mechanics(gell_ensemble* e, int steps, int substeps) {
    GELL_RANGE("gell_ensemble_run_mechanics");
    if (!e || steps < 0 || substeps < 0) return GELL_ERR_INVALID_ARG;
    if (steps == 0) return GELL_OK;
    int left = steps;
    bool graphs = true;
    for (gell_ctx* c : e->m) {
        if (c->prof_on) graphs = false;
        if (!c->stepped) {
            // a context's first step runs outside any capture (first-use set-up of the kernels):
            // every member takes one ordinary step
            for (gell_ctx* d : e->m) {
                if (gell_status st = gell::cells_begin(d)) return st;
                if (gell_status st = gell::cells_end(d, gell::one_mechanics_step(d, substeps))) return st;
                d->stepped = true;
            }
            --left;
            break;
        }
    }
    if (left >= 2 && graphs) {
        if (gell_status st = gather(e)) return st;
        if (!key_matches(e, substeps))
            if (gell_status st = capture(e, substeps)) return st;
        for (; left >= 2; left -= 2) {
            if (cudaGraphLaunch(e->exec, e->origin) != cudaSuccess) {
                cudaGetLastError();
                return GELL_ERR_CUDA;
            }
            for (size_t i = 0; i < e->m.size(); ++i) e->m[i]->launches += e->launches[i];
        }
        if (gell_status st = scatter(e)) return st;
    }
    for (; left > 0; --left)
        for (gell_ctx* c : e->m) {
            if (gell_status st = gell::cells_begin(c)) return st;
            if (gell_status st = gell::one_mechanics_step(c, substeps)) return st;
        }
    for (gell_ctx* c : e->m)
        if (gell_status st = gell::cells_end(c, GELL_OK)) return st;
    return GELL_OK;
}

gell_status gell_ensemble_sync(gell_ensemble* e) {
    if (!e) return GELL_ERR_INVALID_ARG;
    if (cudaStreamSynchronize(e->origin) != cudaSuccess) return GELL_ERR_CUDA;
    for (gell_ctx* c : e->m)
        if (gell_status st = gell_sync(c)) return st;
    return GELL_OK;
}

gell_status gell_ensemble_tune(gell_ensemble* e, int substeps, int* steps_taken, int* best_branches,
                               int* best_sweep_warps) {
    if (!e || substeps < 0) return GELL_ERR_INVALID_ARG;
    int taken = 0;
    // get past every member's first (uncaptured) step
    if (gell_status st = gell_ensemble_run_mechanics(e, 1, substeps)) return st;
    ++taken;
    const int nb = (int)e->pool.size();
    cudaEvent_t t0, t1;
    if (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess) return GELL_ERR_CUDA;
    float best = 3.4e38f;
    int bb = e->branches, bw = e->sweep_warps;
    bool bbat = e->batched;
    gell_status st = GELL_OK;
    for (int v = 0; v < 4; ++v) {
        // line-tile widths 0, 2, 1 with per-member sweeps, then the batched sweeps
        const int w = v == 1 ? 2 : (v == 2 ? 1 : 0);
        e->batched = v == 3;
        for (int b = 1; st == GELL_OK; b *= 2) {
            const int br = b < nb ? b : nb;
            e->branches = br;
            e->sweep_warps = w;
            apply_warps(e);
            st = gather(e);
            if (st == GELL_OK && !key_matches(e, substeps)) st = capture(e, substeps);
            if (st == GELL_OK && cudaGraphUpload(e->exec, e->origin) != cudaSuccess) st = GELL_ERR_CUDA;
            if (st == GELL_OK && (cudaEventRecord(t0, e->origin) != cudaSuccess ||
                                  cudaGraphLaunch(e->exec, e->origin) != cudaSuccess ||
                                  cudaEventRecord(t1, e->origin) != cudaSuccess ||
                                  cudaEventSynchronize(t1) != cudaSuccess))
                st = GELL_ERR_CUDA;
            if (st == GELL_OK) {
                for (size_t i = 0; i < e->m.size(); ++i) e->m[i]->launches += e->launches[i];
                taken += 2;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, t0, t1);
                if (ms < best) {
                    best = ms;
                    bb = br;
                    bw = w;
                    bbat = e->batched;
                }
                st = scatter(e);
            }
            if (br == nb) break;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (st != GELL_OK) {
        cudaGetLastError();
        return st;
    }
    e->branches = bb;
    e->sweep_warps = bw;
    e->batched = bbat;
    apply_warps(e);
    for (gell_ctx* c : e->m)
        if (gell_status s2 = gell::cells_end(c, GELL_OK)) return s2;
    if (steps_taken) *steps_taken = taken;
    if (best_branches) *best_branches = bb;
    if (best_sweep_warps) *best_sweep_warps = bw;
    return GELL_OK;
}

}  // extern "C"
