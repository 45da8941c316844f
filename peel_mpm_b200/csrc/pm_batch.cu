// Batched substep: many independent scenes, packed into one particle array,
// advanced by one launch per kernel over the work of all scenes (one key
// pass, one radix sort, one P2G, one grid update, one G2P).
//
// Packing: scene s owns particles [pb[s], pb[s+1]) of the concatenated planes,
// grid nodes [nodeb[s], nodeb[s] + ng_s^3) of one node buffer, sort blocks
// [sblk[s], sblk[s+1]) of one key space, 4^3 grid blocks [gblk[s], gblk[s+1])
// of one block mask and G2P CTAs [ctab[s], ctab[s+1]).  The scene tables and
// the per-scene parameters live in the workspace, so a captured graph of
// pm_batch_substep calls needs no host data; the host derives launch sizes
// from (n, n_grid) arrays, which must be those the workspace was initialised
// for (checked against a host-side record of each workspace).
#include <cstdint>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "pm_kernels.cuh"

namespace {

using pm::report_error;

struct BatchPlan {
    int S = 0;
    long long n_total = 0, n_nodes = 0, n_gblocks = 0, n_sblocks = 0, n_ctas = 0;
    std::vector<long long> pb, nodeb, sblk, gblk, ctab;
    size_t off_prms = 0, off_pb = 0, off_nodeb = 0, off_sblk = 0, off_gblk = 0, off_ctab = 0;
    pm::Layout L{};
    uint64_t sig = 0;
};

int bits_for(unsigned long long v) {
    int b = 0;
    while ((1ull << b) < v) ++b;
    return b;
}

uint64_t mix(uint64_t h, uint64_t v) {
    h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    return h;
}

int make_plan(int32_t S, const int64_t *n, const int32_t *ng, BatchPlan &bp) {
    if (S < 1 || S > PM_MAX_BATCH_SCENES) return report_error(PM_ERR_ARG, "n_scenes must be in [1, PM_MAX_BATCH_SCENES]");
    if (!n || !ng) return report_error(PM_ERR_ARG, "scene size arrays are NULL");
    bp.S = S;
    bp.pb.assign(S + 1, 0);
    bp.nodeb.assign(S + 1, 0);
    bp.sblk.assign(S + 1, 0);
    bp.gblk.assign(S + 1, 0);
    bp.ctab.assign(S + 1, 0);
    uint64_t h = mix(0, (uint64_t)S);
    for (int s = 0; s < S; ++s) {
        if (n[s] < 0) return report_error(PM_ERR_ARG, "scene particle count < 0");
        if (ng[s] < 4 || ng[s] > 1024) return report_error(PM_ERR_ARG, "scene n_grid must be in [4, 1024]");
        const long long g = ng[s];
        const long long nbs = (g + pm::kBlockEdge - 1) / pm::kBlockEdge;
        const long long nb8 = pm::sort_blocks_per_axis((int)g);
        bp.pb[s + 1] = bp.pb[s] + n[s];
        bp.nodeb[s + 1] = bp.nodeb[s] + g * g * g;
        bp.gblk[s + 1] = bp.gblk[s] + nbs * nbs * nbs;
        bp.sblk[s + 1] = bp.sblk[s] + nb8 * nb8 * nb8;
        bp.ctab[s + 1] = bp.ctab[s] + (n[s] + pm::kG2PThreads - 1) / pm::kG2PThreads;
        h = mix(mix(h, (uint64_t)n[s]), (uint64_t)ng[s]);
    }
    bp.n_total = bp.pb[S];
    bp.n_nodes = bp.nodeb[S];
    bp.n_gblocks = bp.gblk[S];
    bp.n_sblocks = bp.sblk[S];
    bp.n_ctas = bp.ctab[S];
    if (bp.n_total >= (1LL << 31)) return report_error(PM_ERR_ARG, "batch particle count must be < 2^31");
    if (bp.n_gblocks >= (1LL << 31)) return report_error(PM_ERR_ARG, "batch grid is too large");
    const int key_bits = bits_for((unsigned long long)bp.n_sblocks) + pm::kSortBlockBits;
    if (key_bits > 32) return report_error(PM_ERR_ARG, "batch has more than 2^23 sort blocks");
    // tables: params [S], then pb, nodeb, sblk, gblk, ctab as int64 [S + 1] each
    const size_t A = 256, arr = 8 * (size_t)(S + 1);
    size_t o = 0;
    bp.off_prms = o;  o = pm::align_up(o + sizeof(pm_params) * (size_t)S, A);
    bp.off_pb = o;    o = pm::align_up(o + arr, A);
    bp.off_nodeb = o; o = pm::align_up(o + arr, A);
    bp.off_sblk = o;  o = pm::align_up(o + arr, A);
    bp.off_gblk = o;  o = pm::align_up(o + arr, A);
    bp.off_ctab = o;  o = pm::align_up(o + arr, A);
    bp.L = pm::make_layout_sized(bp.n_total, bp.n_nodes, bp.n_gblocks, key_bits, S, o);
    bp.off_prms += bp.L.tables;
    bp.off_pb += bp.L.tables;
    bp.off_nodeb += bp.L.tables;
    bp.off_sblk += bp.L.tables;
    bp.off_gblk += bp.L.tables;
    bp.off_ctab += bp.L.tables;
    bp.sig = mix(h, (uint64_t)bp.L.total);
    return PM_OK;
}

pm::BatchScenes scenes_of(void *ws, const BatchPlan &bp) {
    char *b = (char *)ws;
    pm::BatchScenes sc;
    sc.prms = (const pm_params *)(b + bp.off_prms);
    sc.pb = (const long long *)(b + bp.off_pb);
    sc.nodeb = (const long long *)(b + bp.off_nodeb);
    sc.sblk = (const long long *)(b + bp.off_sblk);
    sc.gblk = (const long long *)(b + bp.off_gblk);
    sc.ctab = (const long long *)(b + bp.off_ctab);
    sc.n = bp.S;
    return sc;
}

// Host record of which batch each workspace was initialised for.
std::mutex g_mu;
struct WsRecord {
    uint64_t sig;
    int p2g_ctas, grid_ctas, stress_ctas, g2p_ctas;   // launch knobs, from the stored parameters of scene 0
};
std::unordered_map<uintptr_t, WsRecord> g_sig;

// Launch knobs recorded for this workspace (0 when none).
WsRecord recorded_knobs(const void *ws) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_sig.find((uintptr_t)ws);
    return it == g_sig.end() ? WsRecord{0, 0, 0, 0, 0} : it->second;
}


int check_ws(void *ws, size_t bytes, const BatchPlan &bp, bool require_record) {
    if (!ws) return report_error(PM_ERR_WORKSPACE, "workspace is NULL");
    if (((uintptr_t)ws & 255) != 0) return report_error(PM_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    if (bytes < bp.L.total) return report_error(PM_ERR_WORKSPACE, "workspace too small for the batch");
    if (require_record) {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_sig.find((uintptr_t)ws);
        if (it == g_sig.end() || it->second.sig != bp.sig)
            return report_error(PM_ERR_WORKSPACE,
                                "workspace was not initialised by pm_batch_workspace_init for these scenes");
    }
    return PM_OK;
}

int upload_tables(void *ws, const BatchPlan &bp, const pm_params *prms, cudaStream_t s) {
    char *b = (char *)ws;
    // pageable source: cudaMemcpyAsync returns once the data is staged, so the
    // caller's arrays (and these vectors) may go away afterwards
    const size_t arr = 8 * (size_t)(bp.S + 1);
    if (cudaMemcpyAsync(b + bp.off_prms, prms, sizeof(pm_params) * (size_t)bp.S, cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(b + bp.off_pb, bp.pb.data(), arr, cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(b + bp.off_nodeb, bp.nodeb.data(), arr, cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(b + bp.off_sblk, bp.sblk.data(), arr, cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(b + bp.off_gblk, bp.gblk.data(), arr, cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(b + bp.off_ctab, bp.ctab.data(), arr, cudaMemcpyHostToDevice, s))
        return pm::api_cuda_check("batch tables");
    // pageable copies are not ordered with later host writes to the source;
    // wait so the vectors can be released
    if (cudaStreamSynchronize(s) != cudaSuccess) return pm::api_cuda_check("batch tables");
    return PM_OK;
}

int plan_from_params(int32_t S, const int64_t *n, const pm_params *prms, BatchPlan &bp) {
    if (!prms) return report_error(PM_ERR_ARG, "params is NULL");
    if (S < 1 || S > PM_MAX_BATCH_SCENES) return report_error(PM_ERR_ARG, "n_scenes must be in [1, PM_MAX_BATCH_SCENES]");
    std::vector<int32_t> ng(S);
    for (int s = 0; s < S; ++s) {
        int rc = pm::api_check_params(prms + s);
        if (rc) return rc;
        ng[s] = prms[s].n_grid;
    }
    return make_plan(S, n, ng.data(), bp);
}

}  // namespace

extern "C" {

int pm_batch_workspace_size(int32_t n_scenes, const int64_t *n, const int32_t *n_grid, size_t *bytes) {
    if (!bytes) return report_error(PM_ERR_ARG, "bytes is NULL");
    BatchPlan bp;
    int rc = make_plan(n_scenes, n, n_grid, bp);
    if (rc) return rc;
    *bytes = bp.L.total;
    return PM_OK;
}

int pm_batch_workspace_layout(int32_t n_scenes, const int64_t *n, const int32_t *n_grid, pm_batch_layout *out) {
    if (!out) return report_error(PM_ERR_ARG, "out is NULL");
    BatchPlan bp;
    int rc = make_plan(n_scenes, n, n_grid, bp);
    if (rc) return rc;
    const pm::Layout &L = bp.L;
    pm_ws_layout &w = out->ws;
    w.ctrl = L.ctrl; w.keys_a = L.keys_a; w.keys_b = L.keys_b; w.vals_a = L.vals_a; w.vals_b = L.vals_b;
    w.hist = L.hist; w.block_mask = L.block_mask; w.block_list = L.block_list; w.g_mom = L.g_mom;
    w.g_dmg = L.g_dmg; w.g_vel = L.g_vel; w.g_gd = L.g_gd; w.payload = L.payload; w.inv_perm = L.inv_perm;
    w.work = L.work; w.total = L.total; w.sort_passes = L.passes; w.n_tiles = L.n_tiles;
    out->params = bp.off_prms;
    out->tables = bp.off_pb;
    out->n_total = bp.n_total;
    out->n_nodes = bp.n_nodes;
    out->n_grid_blocks = bp.n_gblocks;
    out->n_sort_blocks = bp.n_sblocks;
    out->n_g2p_ctas = bp.n_ctas;
    return PM_OK;
}

int pm_batch_workspace_init(void *ws, size_t ws_bytes, int32_t n_scenes, const int64_t *n, const pm_params *prms,
                            void *stream) {
    int rc;
    if ((rc = pm::api_check_device())) return rc;
    BatchPlan bp;
    if ((rc = plan_from_params(n_scenes, n, prms, bp))) return rc;
    if ((rc = check_ws(ws, ws_bytes, bp, false))) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(ws, 0, bp.L.total, s) != cudaSuccess) return pm::api_cuda_check("pm_batch_workspace_init");
    if ((rc = upload_tables(ws, bp, prms, s))) return rc;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_sig[(uintptr_t)ws] = WsRecord{bp.sig, prms[0].p2g_ctas_per_sm, prms[0].grid_ctas_per_sm,
                                        prms[0].stress_ctas_per_sm, prms[0].g2p_ctas_per_sm};
    }
    return pm::api_cuda_check("pm_batch_workspace_init");
}

int pm_batch_set_params(void *ws, size_t ws_bytes, int32_t n_scenes, const int64_t *n, const pm_params *prms,
                        void *stream) {
    int rc;
    if ((rc = pm::api_check_device())) return rc;
    BatchPlan bp;
    if ((rc = plan_from_params(n_scenes, n, prms, bp))) return rc;
    if ((rc = check_ws(ws, ws_bytes, bp, true))) return rc;
    char *b = (char *)ws;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemcpyAsync(b + bp.off_prms, prms, sizeof(pm_params) * (size_t)bp.S, cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return pm::api_cuda_check("pm_batch_set_params");
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_sig[(uintptr_t)ws].p2g_ctas = prms[0].p2g_ctas_per_sm;
        g_sig[(uintptr_t)ws].grid_ctas = prms[0].grid_ctas_per_sm;
        g_sig[(uintptr_t)ws].stress_ctas = prms[0].stress_ctas_per_sm;
        g_sig[(uintptr_t)ws].g2p_ctas = prms[0].g2p_ctas_per_sm;
    }
    return PM_OK;
}

int pm_batch_substep(int32_t n_scenes, const int64_t *n, const int32_t *n_grid, const pm_particles *P, void *ws,
                     size_t ws_bytes, const pm_clock *dev_clocks, void *stream) {
    int rc;
    if ((rc = pm::api_check_device()) || (rc = pm::api_check_particles(P, true))) return rc;
    if (!dev_clocks) return report_error(PM_ERR_ARG, "device clock row is NULL");
    BatchPlan bp;
    if ((rc = make_plan(n_scenes, n, n_grid, bp))) return rc;
    if (P->n != bp.n_total) return report_error(PM_ERR_ARG, "particles.n differs from the sum of scene sizes");
    if ((rc = check_ws(ws, ws_bytes, bp, true))) return rc;
    const pm::WS w = pm::make_ws(ws, bp.L);
    const pm::BatchScenes sc = scenes_of(ws, bp);
    const pm::Parts parts = pm::make_parts(P);
    cudaStream_t s = (cudaStream_t)stream;
    pm::launch_set_clock_batch(sc, w, dev_clocks, s);
    if (bp.n_total > 0) {
        pm::launch_keys(sc, w, parts, s);
        pm::launch_sort(w, bp.n_total, s, w.inv_perm, true);
        const WsRecord knobs = recorded_knobs(ws);
        pm::launch_p2g(sc, parts, w, s, knobs.p2g_ctas, knobs.stress_ctas);
        pm::launch_compact(w, s);
        pm::launch_grid(sc, w, s, knobs.grid_ctas);
        pm::launch_g2p(sc, parts, w, s, bp.n_ctas, knobs.g2p_ctas);
    }
    return pm::api_cuda_check("pm_batch_substep");
}

int pm_batch_read_status(const void *ws, size_t ws_bytes, int32_t n_scenes, const int64_t *n, const int32_t *n_grid,
                         pm_status_info *out, void *stream) {
    int rc;
    if ((rc = pm::api_check_device())) return rc;
    if (!out) return report_error(PM_ERR_ARG, "out is NULL");
    BatchPlan bp;
    if ((rc = make_plan(n_scenes, n, n_grid, bp))) return rc;
    if ((rc = check_ws(const_cast<void *>(ws), ws_bytes, bp, true))) return rc;
    std::vector<pm::Ctrl> c(bp.S);
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemcpyAsync(c.data(), (const char *)ws + bp.L.ctrl, sizeof(pm::Ctrl) * (size_t)bp.S,
                        cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return pm::api_cuda_check("pm_batch_read_status");
    for (int i = 0; i < bp.S; ++i) {
        out[i].nonfinite = c[i].nonfinite;
        out[i].dense_subblocks = c[i].dense_subblocks;
        out[i].n_active_blocks = c[0].n_active;   // one counter for the whole batch
        out[i].any_allow = c[i].any_allow;
    }
    return PM_OK;
}

int pm_batch_workspace_release(const void *ws) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_sig.erase((uintptr_t)ws);
    return PM_OK;
}

}  // extern "C"
