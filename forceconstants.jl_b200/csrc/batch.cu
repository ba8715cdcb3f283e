// Batched snapshots: many LJ snapshots of uneven size through IFC3 assembly,
// mass weighting and full-mode mcc3 as ONE CUDA-graph launch.
//
// The reference computes instantaneous force constants one snapshot at a time
// (third_order → mass_weight_third_order! → CuArray → mcc3, README.md:69-76).
// Here a batch owns device copies of every snapshot's inputs and
//   * admits snapshots into parallel lanes by HBM footprint: each lane is a
//     child context with its own scratch (split operand, two mode-product
//     intermediates, pair tables), sized for its largest snapshot; the number
//     of lanes is what the memory budget allows (at most 4), and snapshots are
//     spread over the lanes largest-work-first;
//   * runs the first fcb200_batch_run eagerly (this sizes every lane's scratch
//     and tunes nothing behind the caller's back), then captures the whole batch
//     — every lane stream forked from and joined back to the caller's stream —
//     into one CUDA graph that later runs replay with a single launch;
//   * keeps Ψ only as the mass-weighted operand of the mode products (the FP64
//     Ψ is assembled in registers and never stored);
//   * uses the mode-tile counts found by fcb200_autotune_mcc3 for each size.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "fcb200_internal.cuh"

namespace fcb {
namespace {

struct Snap {
    int64_t N = 0, n = 0;
    double sigma = 0, eps = 0, r_cut = 0, tol = 0;
    int cap = 0;  // sparse-table capacity (0: dense first mode product)
    Buf pos, box, masses, phi;
    float* k3 = nullptr;
};

size_t snapshot_footprint(int64_t N, int precision, int cap) {
    const int64_t n = 3 * N;
    const size_t pair = (size_t)N * N * (27 * 8 + 1) + (size_t)N * 27 * 8;
    if (precision == FCB_MCC3_FP32) return pair + 3 * sizeof(float) * (size_t)n * n * n;
    const int kind = precision == FCB_MCC3_BF16X3 ? 1 : 2;
    const size_t esz = kind == 1 ? 2 : 4;
    const size_t np = (size_t)pad_for(kind, n);
    if (cap > 0) {  // U1, U2 planes, φ planes, coefficient tables, neighbour lists
        const size_t tables = sizeof(float) * (size_t)N * 27 * 3 * cap + sizeof(int) * (size_t)(N * N + 2 * N + 1);
        if (tc_pair_enabled() && compact_pays(n, n, cap) && sparse_p1c_smem_bytes(cap) <= 227 * 1024) {  // compact U1, per-atom φ rows, padded U2
            const size_t Mp = (size_t)compact_Mp(n), Kc = (size_t)compact_Kc(cap);
            return pair + tables + 2 * esz * (Mp * n * Kc + (size_t)N * n * Kc + Mp * n * n + np * n);
        }
        return pair + tables + 2 * esz * np * (size_t)(2 * n * n + n);
    }
    return pair + 2 * esz * np * (size_t)(3 * n * n + n);
}

// Capacity of the sparse tables for a snapshot: its largest neighbourhood
// (atoms within r_cut + 0.1 Å by the single minimum image, itself included)
// plus 4 atoms of headroom, a multiple of 4; 0 selects the dense first mode
// product (FP32 precision, or tables too large for shared memory).  The
// headroom lets positions move between replays of the captured graph; a
// neighbourhood that outgrows it is reported by the status word.
int host_sparse_cap(const double* pos, int64_t N, const double* box, double r_cut, int precision) {
    if (precision == FCB_MCC3_FP32) return 0;
    const double rc = r_cut + 0.1, rc2 = rc * rc;
    int64_t maxc = 0;
    for (int64_t K = 0; K < N; ++K) {
        int64_t c = 1;
        for (int64_t J = 0; J < N; ++J) {
            if (J == K) continue;
            double d2 = 0.0;
            for (int x = 0; x < 3; ++x) {
                double r = pos[3 * K + x] - pos[3 * J + x];
                if (r > box[x] / 2.0) r -= box[x];
                else if (r < -box[x] / 2.0) r += box[x];
                d2 += r * r;
            }
            if (d2 < rc2) ++c;
        }
        maxc = std::max(maxc, c);
    }
    int64_t cap = (maxc + 4 + 3) / 4 * 4;
    if (cap > N) cap = (N + 3) / 4 * 4;
    if (sparse_p1_smem_bytes((int)cap, N) > 200 * 1024) return 0;
    return (int)cap;
}

fcb200_context* child_context(fcb200_context* parent) {
    auto* c = new fcb200_context();
    c->device = parent->device;
    c->sm_count = parent->sm_count;
    c->d_status = parent->d_status;
    c->tune = parent->tune;
    cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking);
    for (auto& ev : c->ev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    return c;
}

void release_context(fcb200_context* c) {
    Buf* bufs[] = {&c->pos, &c->box, &c->masses, &c->pair_t, &c->pair_flag, &c->self_t, &c->psi_stage, &c->phi_f32,
                   &c->phi_hi, &c->phi_lo, &c->psi_hi, &c->psi_lo, &c->u1_hi, &c->u1_lo, &c->u2_hi, &c->u2_lo,
                   &c->u1_f32, &c->u2_f32, &c->psi_f32, &c->k3_stage[0], &c->k3_stage[1], &c->sp_ints,
                   &c->sp_coef, &c->phik_hi, &c->phik_lo};
    for (Buf* b : bufs) b->release();
    if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
    for (auto& ev : c->ev)
        if (ev) cudaEventDestroy(ev);
    delete c;
}

}  // namespace
}  // namespace fcb

using namespace fcb;

struct fcb200_batch {
    fcb200_context* h = nullptr;
    int precision = FCB_MCC3_BF16X3;
    size_t budget = 0;
    std::vector<Snap*> snaps;
    std::vector<fcb200_context*> lanes;
    std::vector<cudaStream_t> lane_streams;
    std::vector<std::vector<int>> plan;
    std::vector<cudaEvent_t> events;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap = nullptr;  // capture stream (the caller's may be the legacy stream)
    int runs = 0;
    size_t footprint = 0;
    bool dirty = true;
};

namespace {

void drop_graph(fcb200_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

void drop_lanes(fcb200_batch* b) {
    drop_graph(b);
    for (auto* c : b->lanes) release_context(c);
    for (auto s : b->lane_streams) cudaStreamDestroy(s);
    for (auto e : b->events) cudaEventDestroy(e);
    b->lanes.clear();
    b->lane_streams.clear();
    b->events.clear();
    b->plan.clear();
}

int make_plan(fcb200_batch* b) {
    drop_lanes(b);
    size_t maxfp = 0;
    for (auto* s : b->snaps) maxfp = std::max(maxfp, snapshot_footprint(s->N, b->precision, s->cap));
    size_t budget = b->budget;
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        FCB_CUDA(cudaMemGetInfo(&fr, &tot));
        budget = (size_t)(0.8 * (double)fr);
    }
    if (maxfp > budget)
        return set_error(FCB_ERR_OOM, "the largest snapshot needs " + std::to_string(maxfp) +
                                          " bytes of scratch, over the HBM budget of " + std::to_string(budget));
    int L = (int)std::min<size_t>(4, budget / std::max<size_t>(maxfp, 1));
    L = std::max(1, std::min<int>(L, (int)b->snaps.size()));
    // largest work first onto the least loaded lane (work ∝ n⁴)
    std::vector<int> order(b->snaps.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->snaps[x]->n > b->snaps[y]->n; });
    std::vector<double> load(L, 0.0);
    std::vector<size_t> lane_fp(L, 0);
    b->plan.assign(L, {});
    for (int i : order) {
        const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        const double nn = (double)b->snaps[i]->n;
        load[l] += nn * nn * nn * nn;
        lane_fp[l] = std::max(lane_fp[l], snapshot_footprint(b->snaps[i]->N, b->precision, b->snaps[i]->cap));
        b->plan[l].push_back(i);
    }
    b->footprint = 0;
    for (size_t f : lane_fp) b->footprint += f;
    for (int l = 0; l < L; ++l) {
        b->lanes.push_back(child_context(b->h));
        cudaStream_t st;
        FCB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        b->lane_streams.push_back(st);
    }
    b->events.resize(L + 1);
    for (auto& e : b->events) FCB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->dirty = false;
    return FCB_OK;
}

// All snapshots of the batch on the lane streams, forked from / joined to s.
int issue(fcb200_batch* b, cudaStream_t s) {
    FCB_CUDA(cudaEventRecord(b->events[0], s));
    for (size_t l = 0; l < b->lanes.size(); ++l) {
        cudaStream_t ls = b->lane_streams[l];
        FCB_CUDA(cudaStreamWaitEvent(ls, b->events[0], 0));
        for (int i : b->plan[l]) {
            Snap* sn = b->snaps[i];
            if (sn->cap > 0)
                FCB_TRY(snapshot_lj_sparse_device(b->lanes[l], sn->pos.as<double>(), sn->N, sn->box.as<double>(),
                                                  sn->sigma, sn->eps, sn->r_cut, sn->tol, sn->masses.as<double>(),
                                                  sn->phi.as<float>(), 0, sn->n, b->precision, sn->cap, sn->k3, ls));
            else
                FCB_TRY(snapshot_lj_device(b->lanes[l], sn->pos.as<double>(), sn->N, sn->box.as<double>(),
                                           sn->sigma, sn->eps, sn->r_cut, sn->tol, sn->masses.as<double>(),
                                           sn->phi.as<float>(), 0, sn->n, b->precision, sn->k3, ls));
        }
        FCB_CUDA(cudaEventRecord(b->events[l + 1], ls));
        FCB_CUDA(cudaStreamWaitEvent(s, b->events[l + 1], 0));
    }
    return FCB_OK;
}

// ---------------------------------------------------------------- autotune
int autotune_shape(fcb200_context* h, int kind, int64_t n, cudaStream_t s) {
    const int64_t np = pad_for(kind, n);
    const size_t esz = kind == 1 ? 2 : 4;
    FCB_TRY(h->psi_hi.ensure(esz * (size_t)(np * n * n)));
    FCB_TRY(h->psi_lo.ensure(esz * (size_t)(np * n * n)));
    FCB_TRY(h->u1_hi.ensure(esz * (size_t)(np * n * n)));
    FCB_TRY(h->u1_lo.ensure(esz * (size_t)(np * n * n)));
    FCB_TRY(h->phi_hi.ensure(esz * (size_t)(np * n)));
    FCB_TRY(h->phi_lo.ensure(esz * (size_t)(np * n)));
    FCB_CUDA(cudaMemsetAsync(h->psi_hi.p, 0, esz * (size_t)(np * n * n), s));
    FCB_CUDA(cudaMemsetAsync(h->psi_lo.p, 0, esz * (size_t)(np * n * n), s));
    FCB_CUDA(cudaMemsetAsync(h->phi_hi.p, 0, esz * (size_t)(np * n), s));
    FCB_CUDA(cudaMemsetAsync(h->phi_lo.p, 0, esz * (size_t)(np * n), s));
    const ModeProduct mp{n * n, n, n, np, np, n, np, np * n};
    const uint64_t key = tune_key(kind, mp.R, mp.K, mp.M);
    const int lo = (int)((n + 255) / 256), hi = (int)std::min<int64_t>((n + 127) / 128, n);
    cudaEvent_t e0, e1;
    FCB_CUDA(cudaEventCreate(&e0));
    FCB_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int best_nt = lo;
    for (int nt = lo; nt <= hi; ++nt) {
        (*h->tune)[key] = nt;
        int st = mode_product_tc(h, kind, h->psi_hi.p, h->psi_lo.p, h->phi_hi.p, h->phi_lo.p, h->u1_hi.p, h->u1_lo.p,
                                 kind, mp, s);
        if (st != FCB_OK) break;
        cudaEventRecord(e0, s);
        for (int r = 0; r < 3; ++r)
            mode_product_tc(h, kind, h->psi_hi.p, h->psi_lo.p, h->phi_hi.p, h->phi_lo.p, h->u1_hi.p, h->u1_lo.p,
                            kind, mp, s);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms, best_nt = nt;
    }
    (*h->tune)[key] = best_nt;  // P1, P2 and P3 of a full-mode mcc3 share this shape
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return FCB_OK;
}

int load_cache(fcb200_context* h, const char* path) {
    FILE* f = path ? fopen(path, "r") : nullptr;
    if (!f) return FCB_OK;
    char line[256];
    while (fgets(line, sizeof line, f)) {
        unsigned long long key = 0;
        int nt = 0;
        if (sscanf(line, " {\"key\": %llu, \"mode_tiles\": %d", &key, &nt) == 2) (*h->tune)[key] = nt;
    }
    fclose(f);
    return FCB_OK;
}

int save_cache(fcb200_context* h, const char* path) {
    if (!path) return FCB_OK;
    FILE* f = fopen(path, "w");
    if (!f) return set_error(FCB_ERR_ARG, std::string("cannot write autotune cache ") + path);
    fprintf(f, "[\n");
    size_t i = 0;
    for (auto& kv : *h->tune)
        fprintf(f, " {\"key\": %llu, \"mode_tiles\": %d}%s\n", (unsigned long long)kv.first, kv.second,
                ++i < h->tune->size() ? "," : "");
    fprintf(f, "]\n");
    fclose(f);
    return FCB_OK;
}

}  // namespace

extern "C" {

int fcb200_autotune_mcc3(fcb200_handle h, int64_t n, int precision, const char* cache_path, void* stream) {
    if (!h) return set_error(FCB_ERR_ARG, "NULL handle");
    if (n < 16) return set_error(FCB_ERR_ARG, "n must be >= 16");
    if (precision != FCB_MCC3_BF16X3 && precision != FCB_MCC3_TF32X3) return FCB_OK;  // FP32 SIMT has fixed tiles
    cudaSetDevice(h->device);
    if (!h->tune) {
        h->tune = new std::unordered_map<uint64_t, int>();
        h->owns_tune = true;
    }
    FCB_TRY(load_cache(h, cache_path));
    const int kind = precision == FCB_MCC3_BF16X3 ? 1 : 2;
    const int64_t np = pad_for(kind, n);
    if (h->tune->count(tune_key(kind, n * n, n, n)) == 0) {
        (void)np;
        FCB_TRY(autotune_shape(h, kind, n, static_cast<cudaStream_t>(stream)));
        FCB_TRY(save_cache(h, cache_path));
    }
    return FCB_OK;
}

int fcb200_batch_create(fcb200_handle h, int precision, size_t hbm_budget_bytes, fcb200_batch_t* out) {
    if (!h || !out) return set_error(FCB_ERR_ARG, "NULL argument");
    if (precision != FCB_MCC3_FP32 && precision != FCB_MCC3_BF16X3 && precision != FCB_MCC3_TF32X3)
        return set_error(FCB_ERR_ARG, "unknown mcc3 precision mode");
    auto* b = new fcb200_batch();
    b->h = h;
    b->precision = precision;
    b->budget = hbm_budget_bytes;
    *out = b;
    return FCB_OK;
}

int fcb200_batch_add_lj(fcb200_batch_t b, const double* pos, int64_t N, const double* box, double sigma, double eps,
                        double r_cut, double tol, const double* masses, const float* phi, float* k3_out) {
    if (!b) return set_error(FCB_ERR_ARG, "NULL batch");
    if (!pos || !box || !masses || !phi || !k3_out) return set_error(FCB_ERR_ARG, "NULL input or output");
    if (N < 1 || N > 4096) return set_error(FCB_ERR_ARG, "n_atoms out of range");
    if (!is_device_ptr(k3_out)) return set_error(FCB_ERR_ARG, "k3_out must be device memory for a batch");
    double bh[3];
    if (is_device_ptr(box)) {
        FCB_CUDA(cudaMemcpy(bh, box, sizeof bh, cudaMemcpyDeviceToHost));
    } else {
        for (int d = 0; d < 3; ++d) bh[d] = box[d];
    }
    for (int d = 0; d < 3; ++d)
        if (!(r_cut < bh[d])) return set_error(FCB_ERR_CUTOFF, "Cutoff larger than L/2 (r_cut must be < box length)");
    cudaSetDevice(b->h->device);
    auto* s = new Snap();
    s->N = N;
    s->n = 3 * N;
    s->sigma = sigma;
    s->eps = eps;
    s->r_cut = r_cut;
    s->tol = tol;
    s->k3 = k3_out;
    int st = FCB_OK;
    if ((st = s->pos.ensure(sizeof(double) * 3 * N)) || (st = s->box.ensure(sizeof(double) * 3)) ||
        (st = s->masses.ensure(sizeof(double) * N)) || (st = s->phi.ensure(sizeof(float) * s->n * s->n))) {
        delete s;
        return st;
    }
    FCB_CUDA(cudaMemcpy(s->pos.p, pos, sizeof(double) * 3 * N, cudaMemcpyDefault));
    {
        std::vector<double> hp((size_t)(3 * N));
        FCB_CUDA(cudaMemcpy(hp.data(), pos, sizeof(double) * 3 * N, cudaMemcpyDefault));
        s->cap = host_sparse_cap(hp.data(), N, bh, r_cut, b->precision);
    }
    FCB_CUDA(cudaMemcpy(s->box.p, bh, sizeof(double) * 3, cudaMemcpyHostToDevice));
    FCB_CUDA(cudaMemcpy(s->masses.p, masses, sizeof(double) * N, cudaMemcpyDefault));
    FCB_CUDA(cudaMemcpy(s->phi.p, phi, sizeof(float) * s->n * s->n, cudaMemcpyDefault));
    b->snaps.push_back(s);
    b->dirty = true;
    return FCB_OK;
}

int fcb200_batch_set_positions(fcb200_batch_t b, int64_t index, const double* pos, void* stream) {
    if (!b || index < 0 || index >= (int64_t)b->snaps.size() || !pos) return set_error(FCB_ERR_ARG, "bad argument");
    Snap* s = b->snaps[index];
    if (s->cap > 0) {
        // a neighbourhood past the sparse tables' capacity re-plans the batch
        std::vector<double> hp((size_t)(3 * s->N));
        double bh[3];
        FCB_CUDA(cudaMemcpy(hp.data(), pos, sizeof(double) * 3 * s->N, cudaMemcpyDefault));
        FCB_CUDA(cudaMemcpy(bh, s->box.p, sizeof bh, cudaMemcpyDeviceToHost));
        const int cap = host_sparse_cap(hp.data(), s->N, bh, s->r_cut, b->precision);
        if (cap == 0 || cap > s->cap) {
            s->cap = cap;
            b->dirty = true;
        }
    }
    FCB_CUDA(cudaMemcpyAsync(s->pos.p, pos, sizeof(double) * 3 * s->N, cudaMemcpyDefault,
                             static_cast<cudaStream_t>(stream)));
    return FCB_OK;
}

int fcb200_batch_run(fcb200_batch_t b, void* stream) {
    if (!b) return set_error(FCB_ERR_ARG, "NULL batch");
    if (b->snaps.empty()) return FCB_OK;
    cudaSetDevice(b->h->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (b->dirty) {
        FCB_TRY(make_plan(b));
        b->runs = 0;
    }
    if (b->runs == 0) {
        // eager pass: allocates every lane's scratch at its largest size
        FCB_TRY(issue(b, s));
        ++b->runs;
        return FCB_OK;
    }
    if (!b->exec) {
        if (!b->cap) FCB_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
        FCB_CUDA(cudaStreamSynchronize(s));
        FCB_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeRelaxed));
        int st = issue(b, b->cap);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->cap, &g);
        if (st != FCB_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture(batch)");
        b->graph = g;
        FCB_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
    }
    FCB_CUDA(cudaGraphLaunch(b->exec, s));
    ++b->runs;
    return FCB_OK;
}

int fcb200_batch_info(fcb200_batch_t b, int64_t* n_snapshots, int64_t* lanes, int64_t* graph_nodes,
                      size_t* scratch_bytes) {
    if (!b) return set_error(FCB_ERR_ARG, "NULL batch");
    if (n_snapshots) *n_snapshots = (int64_t)b->snaps.size();
    if (lanes) *lanes = (int64_t)b->lanes.size();
    if (graph_nodes) {
        size_t nn = 0;
        if (b->graph) cudaGraphGetNodes(b->graph, nullptr, &nn);
        *graph_nodes = (int64_t)nn;
    }
    if (scratch_bytes) *scratch_bytes = b->footprint;
    return FCB_OK;
}

int fcb200_batch_lane(fcb200_batch_t b, int64_t index, int64_t* lane) {
    if (!b || !lane || index < 0 || index >= (int64_t)b->snaps.size()) return set_error(FCB_ERR_ARG, "bad argument");
    if (b->dirty || b->plan.empty())
        return set_error(FCB_ERR_ARG, "the batch has no plan yet: fcb200_batch_run makes it");
    for (size_t l = 0; l < b->plan.size(); ++l)
        for (int i : b->plan[l])
            if (i == index) {
                *lane = (int64_t)l;
                return FCB_OK;
            }
    return set_error(FCB_ERR_ARG, "snapshot not in the plan");
}

int fcb200_batch_destroy(fcb200_batch_t b) {
    if (!b) return FCB_OK;
    cudaSetDevice(b->h->device);
    cudaDeviceSynchronize();
    drop_lanes(b);
    if (b->cap) cudaStreamDestroy(b->cap);
    for (auto* s : b->snaps) {
        s->pos.release();
        s->box.release();
        s->masses.release();
        s->phi.release();
        delete s;
    }
    delete b;
    return FCB_OK;
}

}  // extern "C"
