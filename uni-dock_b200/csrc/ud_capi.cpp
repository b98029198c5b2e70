// C ABI of the engine (include/unidock_b200.h): handle management, host <->
// device marshalling, batch scheduling and result post-processing.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iomanip>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/unidock_b200.h"
#include "ud_engine.h"
#include "ud_model.h"

static_assert(ud::kAd4TableRowElec == ud::kAd4RowElec && ud::kAd4TableRowDesolv == ud::kAd4RowDesolv,
              "AD4 table layout shared by host and device");
static_assert(ud::kAdTypes == ud::AD_SIZE, "AD4 parameter arrays cover every AD type");


using namespace ud;

namespace {

thread_local std::string g_error;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw Error(UD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorName(e) + " " + cudaGetErrorString(e));
}

template <class T> struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    // Grows with a quarter of headroom: a batch handle reused for batches of
    // similar size then never reallocates, and a free (cudaFree synchronises
    // the whole device) never stalls the host behind another stream's search.
    void alloc(size_t count) {
        if (count <= n && p) return;
        release();
        const size_t cap = std::max<size_t>(count + count / 4, 1);
        cuda_check(cudaMalloc(&p, cap * sizeof(T)), "cudaMalloc");
        n = cap;
    }
    void upload(const T* src, size_t count, cudaStream_t s) {
        alloc(count);
        if (count) cuda_check(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, s), "H2D");
    }
};

// Page-locked host buffer (device-to-host copies of a captured search graph).
template <class T> struct PinnedBuf {
    T* p = nullptr;
    size_t n = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
    void alloc(size_t count) {  // with headroom, as DevBuf::alloc (cudaFreeHost synchronises too)
        if (count <= n && p) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        const size_t cap = std::max<size_t>(count + count / 4, 1);
        cuda_check(cudaMallocHost((void**)&p, cap * sizeof(T)), "cudaMallocHost");
        n = cap;
    }
};

template <class F> int guarded(F&& f) {
    try {
        f();
        return UD_OK;
    } catch (const Error& e) {
        g_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_error = e.what();
        return UD_ERR_PARSE;
    } catch (...) {
        g_error = "unknown error";
        return UD_ERR_ARG;
    }
}

}  // namespace

// Pair tables of a scoring function (all terms weighted, or one term
// unweighted), built once per process for each (function, weights, term):
// building one takes tens of milliseconds of host time, and screens with
// many receptors (paired batches) create many maps with the same function.
static std::shared_ptr<const PairTable> cached_table(const Scoring& sf, int term = -1) {
    static std::mutex mu;
    static std::map<std::string, std::shared_ptr<const PairTable>> cache;
    std::string key = std::to_string(sf.choice) + ' ' + std::to_string(term) + ' ' + std::to_string(sf.cutoff);
    for (float w : sf.weights) key += ' ' + std::to_string(w);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    auto t = std::make_shared<PairTable>();
    t->build(sf, term);
    std::lock_guard<std::mutex> lock(mu);
    return cache.emplace(key, std::move(t)).first->second;
}

struct ud_maps_s {
    Scoring sf;
    MapsDesc desc{};
    std::vector<int> slot_types;     // XS type of each map slot
    DevBuf<float> maps;              // [slot][z][y][x]
    DevBuf<float2> xpairs;           // [slot][z][y][x] = (map at x, map at x + 1): the search's corner loads
    DevBuf<float> smooth;            // [tp][bin][2]
    DevBuf<float> fast;              // [tp][bin]
    int n_bins = 0;
    float factor = 32.0f;
    float cutoff2 = 64.0f;
    // typed receptor atoms (x, y, z, xs as int bits), kept to build term maps
    std::vector<float> rec_xyzt;
    // AD4: receptor atoms (x, y, z, charge) and AD types
    std::vector<float> rec_xyzq;
    std::vector<int> rec_ad;
    // per-term data of weight gradients, built on first use
    DevBuf<float> term_maps;         // [term][slot][z][y][x]
    DevBuf<float> term_rows;         // [term][tp][bin][4], as `smooth`
    DevBuf<float> term_fast;         // [term][tp][bin], as `fast`
    bool terms_built = false;
    bool loaded = false;             // read from map files: no receptor to rebuild per-term maps from
    float box_center[3] = {0, 0, 0}; // box as given (written to map file headers)
    float box_spacing = 0;
    // bias wells added to the maps (and to receptor-atom scoring)
    std::vector<BiasElement> bias;
    DevBuf<BiasRec> d_bias;
    // receptor atoms in box cells for scoring without the maps, built on first use
    DevBuf<float> rc_atoms;
    DevBuf<int> rc_start;
    DeviceReceptorView rc{};
    bool rc_built = false;
};

struct LigandPost {
    std::vector<PoseResult> modes;
};

struct ud_ligand_s {
    Ligand lig;
    // pair-group slots of the Vina / Vinardo and the AD4 pair lists (-1 until
    // counted; memory estimates only, which may run on several threads)
    mutable std::atomic<int> pair_slots[2] = {-1, -1};
};

struct ud_batch_s {
    ud_maps maps = nullptr;
    std::vector<const Ligand*> ligs;
    std::vector<LigDesc> desc;
    DevBuf<LigDesc> d_desc;
    DevBuf<AtomRec> d_atoms;
    DevBuf<NodeRec> d_nodes;
    DevBuf<uint32_t> d_pairs;
    DevBuf<uint32_t> d_grid;
    size_t upload_bytes = 0;  // host-to-device bytes of the last topology fill
    DevBuf<float> d_charge;          // AD4: atom charges
    DevBuf<float> d_pair_coef;       // AD4: (q_a q_b, |q_a| V_b + |q_b| V_a) per pair slot
    int max_atoms = 0, max_tors = 0;
    // search state
    DevBuf<int> d_order;
    DevBuf<unsigned int> d_queue;
    DevBuf<float> d_poses;
    DevBuf<ChainResult> d_results;
    std::vector<float> h_poses;
    std::vector<ChainResult> h_results;
    int pose_stride = 0;
    int exhaustiveness = 0;
    bool searched = false;
    bool launched = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // around the search kernel alone inside the captured graph (event record
    // nodes), so that its own device time is known without a separate launch
    cudaEvent_t evk0 = nullptr, evk1 = nullptr;
    long long evals = 0;
    float kernel_ms = 0;
    std::vector<LigandPost> post;
    std::vector<std::string> text[2];  // rendered output per ligand (PDBQT, SDF), filled on first request
    bool text_ready[2] = {false, false};
    ud_search_params params{};
    // scoring scratch
    DevBuf<int> d_pose_lig;
    DevBuf<float> d_pose;
    DevBuf<float> d_e, d_g, d_score, d_dw;

    // captured per-batch search sequence (use_graph): queue reset, persistent
    // search kernel and the copies of its results into page-locked memory
    cudaStream_t capture_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    std::string graph_key;
    PinnedBuf<float> hp_poses;
    PinnedBuf<ChainResult> hp_results;
    bool graph_results = false;
    // per-ligand bias wells for receptor-atom scoring (multi-bias), all lists
    // back to back; span per ligand: offset | count << 16
    std::vector<std::vector<BiasRec>> lig_bias;
    DevBuf<BiasRec> d_lig_bias;
    DevBuf<int> d_lig_bias_span;
    bool lig_bias_dirty = false;
    // modes of the last search: clustered (and refined) on the device
    int mode_cap = 0;
    bool refined = false;
    DevBuf<float> d_cluster_scratch;
    DevBuf<int> d_n_modes, d_mode_chain, d_mode_lig;
    DevBuf<float> d_mode_pose, d_mode_e;
    PinnedBuf<int> hp_n_modes, hp_mode_chain;
    PinnedBuf<float> hp_mode_pose, hp_mode_e;
    // launch configuration picked by ud_autotune for this batch
    bool tuned = false;
    int tuned_chains_per_block = 4;
    int tuned_lanes_per_chain = 32;
    int tuned_bfgs_cap = 0;

    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        graph_exec = nullptr;
        graph = nullptr;
        graph_key.clear();
    }
    ~ud_batch_s() {
        drop_graph();
        if (capture_stream) cudaStreamDestroy(capture_stream);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (evk0) cudaEventDestroy(evk0);
        if (evk1) cudaEventDestroy(evk1);
    }
    DeviceBatchView view() const {
        return DeviceBatchView{d_desc.p, d_atoms.p, d_nodes.p, d_pairs.p, d_grid.p, max_atoms, max_tors,
                               d_charge.p, d_pair_coef.p, maps && maps->desc.ad4 ? 1 : 0};
    }
};

static DeviceMapsView maps_view(const ud_maps_s* m) { return DeviceMapsView{m->maps.p, m->desc, m->xpairs.p}; }

// The x-pair copy of the maps, rebuilt after every change to the maps.
static void refresh_xpairs(ud_maps_s* m, cudaStream_t s) {
    const size_t n = (size_t)m->desc.dims[0] * m->desc.dims[1] * m->desc.dims[2] * std::max(1, m->desc.n_maps);
    m->xpairs.alloc(n);
    if (m->desc.n_maps > 0) cuda_check(launch_map_xpairs(m->maps.p, m->desc, m->xpairs.p, s), "map x-pairs");
}
static DeviceTablesView tables_view(const ud_maps_s* m) {
    return DeviceTablesView{m->smooth.p, m->fast.p, m->n_bins, m->factor, m->cutoff2};
}

// ---------------------------------------------------------------- receptor

extern "C" int ud_version(void) { return 100; }
extern "C" const char* ud_last_error(void) { return g_error.c_str(); }

extern "C" int ud_receptor_parse(const char* pdbqt, size_t len, float* xyz, int* xs, int capacity,
                                 int* n_atoms) {
    return guarded([&] {
        if (!pdbqt || !n_atoms) throw Error(UD_ERR_ARG, "null argument");
        Receptor R = parse_receptor_pdbqt(std::string(pdbqt, len));
        *n_atoms = (int)R.xyz.size();
        if (xyz || xs) {
            if (capacity < (int)R.xyz.size()) throw Error(UD_ERR_CAPACITY, "receptor capacity too small");
            for (size_t i = 0; i < R.xyz.size(); ++i) {
                if (xyz)
                    for (int k = 0; k < 3; ++k) xyz[3 * i + k] = R.xyz[i][k];
                if (xs) xs[i] = R.xs[i];
            }
        }
    });
}

extern "C" int ud_receptor_parse_ex(const char* pdbqt, size_t len, float* xyz, int* xs, int* ad, float* charge,
                                    int capacity, int* n_atoms) {
    return guarded([&] {
        if (!pdbqt || !n_atoms) throw Error(UD_ERR_ARG, "null argument");
        Receptor R = parse_receptor_pdbqt(std::string(pdbqt, len));
        *n_atoms = (int)R.xyz.size();
        if (xyz || xs || ad || charge) {
            if (capacity < (int)R.xyz.size()) throw Error(UD_ERR_CAPACITY, "receptor capacity too small");
            for (size_t i = 0; i < R.xyz.size(); ++i) {
                if (xyz)
                    for (int k = 0; k < 3; ++k) xyz[3 * i + k] = R.xyz[i][k];
                if (xs) xs[i] = R.xs[i];
                if (ad) ad[i] = R.ad[i];
                if (charge) charge[i] = R.charge[i];
            }
        }
    });
}

// ---------------------------------------------------------------- maps

static std::vector<int> default_map_types() {
    // Vina batch mode computes all XS types of the scoring function with CG
    // folded onto C_H/C_P and glue types skipped (cache.cpp:476-505).
    std::vector<int> t;
    for (int i = 0; i < XS_SIZE; ++i) {
        int g = xs_grid_type(i);
        if (g >= 0 && std::find(t.begin(), t.end(), g) == t.end()) t.push_back(g);
    }
    return t;
}

static size_t round4(size_t n) { return (n + 3) & ~(size_t)3; }

// Lerp rows with both bracketing bins in one 16-byte record:
// [tp][bin] = (e_bin, dor_bin, e_bin+1, dor_bin+1).
static void pack_smooth4(const PairTable& tab, float* s4) {
    const size_t ntp = tab.smooth.size() / (2 * (size_t)tab.n);
    for (size_t tp = 0; tp < ntp; ++tp)
        for (int k = 0; k < tab.n; ++k) {
            const float* row = &tab.smooth[tp * tab.n * 2];
            float* o = &s4[(tp * tab.n + k) * 4];
            o[0] = row[2 * k];
            o[1] = row[2 * k + 1];
            o[2] = (k + 1 < tab.n) ? row[2 * (k + 1)] : 0.0f;
            o[3] = (k + 1 < tab.n) ? row[2 * (k + 1) + 1] : 0.0f;
        }
}

// Receptor-type-major table of the map kernel: [t1][bin][slot].
static void pack_fastT(const PairTable& tab, const std::vector<int>& slot_types, int nslot_pad, float* fastT) {
    for (int t1 = 0; t1 < XS_SIZE; ++t1)
        for (size_t k = 0; k < slot_types.size(); ++k) {
            const float* row = &tab.fast[(size_t)tri_index(t1, slot_types[k]) * tab.n];
            for (int b = 0; b < tab.n; ++b) fastT[((size_t)t1 * tab.n + b) * nslot_pad + k] = row[b];
        }
}

extern "C" int ud_maps_create(int sf, const float* weights, int n_weights, const float* rec_xyz,
                              const int* rec_xs, int n_rec, const float center[3], const float size[3],
                              float spacing, const int* types, int n_types, void* stream, ud_maps* out) {
    return guarded([&] {
        if (!out || !center || !size || (n_rec > 0 && (!rec_xyz || !rec_xs)) || spacing <= 0)
            throw Error(UD_ERR_ARG, "invalid maps arguments");
        if (sf != UD_SF_VINA && sf != UD_SF_VINARDO)
            throw Error(UD_ERR_ARG, "grid maps are built for Vina or Vinardo scoring");
        for (int i = 0; i < 3; ++i)
            if (!(size[i] > 0)) throw Error(UD_ERR_ARG, "box size must be positive");
        cudaStream_t s = (cudaStream_t)stream;
        auto m = std::make_unique<ud_maps_s>();
        std::vector<float> w;
        if (weights && n_weights > 0) {
            w.assign(weights, weights + n_weights);
            // rotatable weight given raw: store 5*w/0.1-1 (vina.cpp:392-432)
            w.back() = (float)(5 * (double)w.back() / 0.1 - 1);
        }
        m->sf = Scoring::make(sf, w.empty() ? nullptr : w.data(), (int)w.size());
        // box (vina.cpp:528-539) and grid frame (grid.cpp:25-38)
        MapsDesc& d = m->desc;
        for (int i = 0; i < 3; ++i) m->box_center[i] = center[i];
        m->box_spacing = spacing;
        for (int i = 0; i < 3; ++i) {
            size_t nvox = (size_t)std::ceil((float)size[i] / (float)spacing);
            float real_span = (float)spacing * nvox;
            float begin = (float)center[i] - real_span / 2;
            float end = begin + real_span;
            d.dims[i] = (int)nvox + 1;
            d.init[i] = begin;
            d.corner2[i] = end;
            float range = end - begin;
            d.dim_m1[i] = (float)(d.dims[i] - 1);
            d.factor[i] = d.dim_m1[i] / range;
            d.factor_inv[i] = 1 / d.factor[i];
        }
        d.slope = 1e6f;
        std::vector<int> req = types && n_types > 0 ? std::vector<int>(types, types + n_types) : default_map_types();
        for (int t : req) {
            int g = xs_grid_type(t);
            if (g < 0) continue;
            if (std::find(m->slot_types.begin(), m->slot_types.end(), g) == m->slot_types.end())
                m->slot_types.push_back(g);
        }
        if (m->slot_types.size() > 36) throw Error(UD_ERR_ARG, "too many map types");
        std::fill(d.slot_of_xs, d.slot_of_xs + 36, (int8_t)-1);
        for (size_t k = 0; k < m->slot_types.size(); ++k) d.slot_of_xs[m->slot_types[k]] = (int8_t)k;
        d.n_maps = (int)m->slot_types.size();
        // pair tables of the scoring function
        const PairTable& tab = *cached_table(m->sf);
        m->n_bins = tab.n;
        m->factor = tab.factor;
        m->cutoff2 = m->sf.cutoff * m->sf.cutoff;
        {
            std::vector<float> s4(tab.smooth.size() * 2, 0.0f);
            pack_smooth4(tab, s4.data());
            m->smooth.upload(s4.data(), s4.size(), s);
        }
        // padded to whole float4s: ud_maps_set_weights rewrites these in place
        m->fast.alloc(round4(tab.fast.size()));
        m->fast.upload(tab.fast.data(), tab.fast.size(), s);
        const int nslot = d.n_maps, nslot_pad = std::max(4, (nslot + 3) & ~3);
        std::vector<float> fastT((size_t)XS_SIZE * tab.n * nslot_pad, 0.0f);
        pack_fastT(tab, m->slot_types, nslot_pad, fastT.data());
        DevBuf<float> d_fastT;
        d_fastT.upload(fastT.data(), fastT.size(), s);
        std::vector<float> rec;
        rec.reserve(4 * (size_t)n_rec);
        for (int i = 0; i < n_rec; ++i) {
            if (rec_xs[i] < 0 || rec_xs[i] >= XS_SIZE) continue;  // untyped atoms contribute nothing
            rec.push_back(rec_xyz[3 * i]);
            rec.push_back(rec_xyz[3 * i + 1]);
            rec.push_back(rec_xyz[3 * i + 2]);
            int t = rec_xs[i];
            float tf;
            std::memcpy(&tf, &t, 4);
            rec.push_back(tf);
        }
        DevBuf<float> d_rec;
        d_rec.upload(rec.data(), rec.size(), s);
        m->rec_xyzt = rec;
        const size_t plane = (size_t)d.dims[0] * d.dims[1] * d.dims[2];
        m->maps.alloc(round4(plane * std::max(1, nslot)));
        if (nslot > 0) {
            cuda_check(launch_maps(d_rec.p, (int)(rec.size() / 4), d_fastT.p, tab.n, nslot, nslot_pad,
                                   tab.factor, m->cutoff2, d, m->maps.p, s),
                       "maps kernel");
        }
        refresh_xpairs(m.get(), s);
        cuda_check(cudaStreamSynchronize(s), "maps sync");
        *out = m.release();
    });
}

// ---------------------------------------------------------------- AD4 maps

// AutoDock 4.2 atom-kind parameters for the map kernel (atom_constants.h).
static Ad4Params ad4_params() {
    Ad4Params P{};
    for (int t = 0; t < AD_SIZE; ++t) {
        const AdKind& k = ad_kind(t);
        P.radius[t] = k.radius;
        P.depth[t] = k.depth;
        P.hb_depth[t] = k.hb_depth;
        P.hb_radius[t] = k.hb_radius;
        P.solvation[t] = ad4_solvation(t);
        P.volume[t] = ad4_volume(t);
    }
    return P;
}

// Map set of AD4 maps `m` with the term weights (term >= 0: that term alone at weight 1).
static Ad4MapSpec ad4_spec(const ud_maps_s* m, int term) {
    Ad4MapSpec S{};
    S.n_slots = m->desc.n_maps - 2;
    for (int k = 0; k < S.n_slots; ++k) S.slot_ad[k] = m->slot_types[k];
    auto w = [&](int t) { return term < 0 ? m->sf.weights[t] : (term == t ? 1.0f : 0.0f); };
    S.w_vdw = w(0);
    S.w_hb = w(1);
    S.w_elec = w(2);
    S.w_dsolv = w(3);
    return S;
}

// AD types an AD4 map set covers by default: every AD kind an atom can read
// (CG carbons read C, glue atoms none, W never occurs in ligands).
static std::vector<int> default_ad4_types() {
    std::vector<int> t;
    for (int a = 0; a < AD_SIZE; ++a)
        if ((a < AD_G0 || a > AD_CG3) && a != AD_W) t.push_back(a);
    return t;
}

extern "C" int ud_maps_create_ad4(const float* weights, int n_weights, const float* rec_xyz, const int* rec_ad,
                                  const float* rec_q, int n_rec, const float center[3], const float size[3],
                                  float spacing, const int* types, int n_types, void* stream, ud_maps* out) {
    return guarded([&] {
        if (!out || !center || !size || (n_rec > 0 && (!rec_xyz || !rec_ad || !rec_q)) || spacing <= 0)
            throw Error(UD_ERR_ARG, "invalid maps arguments");
        for (int i = 0; i < 3; ++i)
            if (!(size[i] > 0)) throw Error(UD_ERR_ARG, "box size must be positive");
        cudaStream_t s = (cudaStream_t)stream;
        auto m = std::make_unique<ud_maps_s>();
        // AD4 weights: vdW, H-bond, electrostatics, desolvation, glue, torsional (raw, ad4_tors_add)
        m->sf = Scoring::make(SF_AD42, (weights && n_weights > 0) ? weights : nullptr,
                              (weights && n_weights > 0) ? n_weights : 0);
        MapsDesc& d = m->desc;
        for (int i = 0; i < 3; ++i) {
            // AutoGrid maps have an even number of voxels per axis (ad4cache.cpp:355-364)
            size_t nvox = (size_t)std::ceil((float)size[i] / (float)spacing);
            if (nvox % 2 == 1) ++nvox;
            // the frame the map reader derives from CENTER and SPACING, so that
            // written maps read back onto the same grid
            const float halfspan = (float)((double)((int)nvox * spacing) / 2.0);
            float begin = (float)center[i] - halfspan;
            float end = (float)center[i] + halfspan;
            m->box_center[i] = center[i];
            d.dims[i] = (int)nvox + 1;
            d.init[i] = begin;
            d.corner2[i] = end;
            d.dim_m1[i] = (float)(d.dims[i] - 1);
            d.factor[i] = d.dim_m1[i] / (end - begin);
            d.factor_inv[i] = 1 / d.factor[i];
        }
        m->box_spacing = spacing;
        d.slope = 1e6f;
        d.ad4 = 1;
        std::vector<int> req = types && n_types > 0 ? std::vector<int>(types, types + n_types) : default_ad4_types();
        for (int t : req) {
            if (t < 0 || t >= AD_SIZE) throw Error(UD_ERR_ARG, "AD type out of range");
            int g = (t >= AD_CG0 && t <= AD_CG3) ? AD_C : t;
            if (g >= AD_G0 && g <= AD_G3) continue;
            if (std::find(m->slot_types.begin(), m->slot_types.end(), g) == m->slot_types.end())
                m->slot_types.push_back(g);
        }
        if (m->slot_types.size() > 34) throw Error(UD_ERR_ARG, "too many map types");
        std::fill(d.slot_of_xs, d.slot_of_xs + 36, (int8_t)-1);
        for (size_t k = 0; k < m->slot_types.size(); ++k) d.slot_of_xs[m->slot_types[k]] = (int8_t)k;
        d.e_slot = (int)m->slot_types.size();
        d.d_slot = d.e_slot + 1;
        d.n_maps = d.d_slot + 1;
        // pair tables: AD type pairs + the shared electrostatic / desolvation rows
        const PairTable& tab = *cached_table(m->sf);
        m->n_bins = tab.n;
        m->factor = tab.factor;
        m->cutoff2 = m->sf.cutoff * m->sf.cutoff;
        {
            std::vector<float> s4(tab.smooth.size() * 2, 0.0f);
            pack_smooth4(tab, s4.data());
            m->smooth.upload(s4.data(), s4.size(), s);
        }
        m->fast.alloc(round4(tab.fast.size()));
        m->fast.upload(tab.fast.data(), tab.fast.size(), s);
        for (int i = 0; i < n_rec; ++i) {
            if (rec_ad[i] < 0 || rec_ad[i] >= AD_SIZE) continue;  // untyped atoms contribute nothing
            for (int k = 0; k < 3; ++k) m->rec_xyzq.push_back(rec_xyz[3 * i + k]);
            m->rec_xyzq.push_back(rec_q[i]);
            m->rec_ad.push_back(rec_ad[i]);
        }
        DevBuf<float> d_rec;
        DevBuf<int> d_ad;
        d_rec.upload(m->rec_xyzq.data(), m->rec_xyzq.size(), s);
        d_ad.upload(m->rec_ad.data(), m->rec_ad.size(), s);
        const size_t plane = (size_t)d.dims[0] * d.dims[1] * d.dims[2];
        m->maps.alloc(round4(plane * d.n_maps));
        cuda_check(launch_maps_ad4(d_rec.p, d_ad.p, (int)m->rec_ad.size(), ad4_params(), ad4_spec(m.get(), -1), d,
                                   m->maps.p, s),
                   "AD4 maps kernel");
        refresh_xpairs(m.get(), s);
        cuda_check(cudaStreamSynchronize(s), "maps sync");
        *out = m.release();
    });
}

// AutoGrid .map files of the maps (header of ad4cache::write, ad4cache.cpp:439-521;
// values at full float precision): AD4 maps as <prefix>.<AD type>.map,
// <prefix>.e.map and <prefix>.d.map; Vina maps as <prefix>.<XS type>.map.
extern "C" int ud_maps_write(ud_maps maps, const char* prefix) {
    return guarded([&] {
        if (!maps || !prefix) throw Error(UD_ERR_ARG, "null argument");
        const MapsDesc& d = maps->desc;
        const size_t plane = (size_t)d.dims[0] * d.dims[1] * d.dims[2];
        std::vector<float> h(plane);
        for (int k = 0; k < d.n_maps; ++k) {
            std::string name;
            if (d.ad4) name = k == d.e_slot ? "e" : k == d.d_slot ? "d" : ad_kind(maps->slot_types[k]).name;
            else name = xs_name(maps->slot_types[k]);
            cuda_check(cudaMemcpy(h.data(), maps->maps.p + plane * k, plane * sizeof(float), cudaMemcpyDeviceToHost),
                       "map D2H");
            std::string path = std::string(prefix) + "." + name + ".map";
            FILE* f = std::fopen(path.c_str(), "w");
            if (!f) throw Error(UD_ERR_ARG, "cannot write " + path);
            std::fprintf(f, "GRID_PARAMETER_FILE NULL\nGRID_DATA_FILE NULL\nMACROMOLECULE NULL\n");
            std::fprintf(f, "SPACING %.9g\n", maps->box_spacing);
            std::fprintf(f, "NELEMENTS %d %d %d\n", d.dims[0] - 1, d.dims[1] - 1, d.dims[2] - 1);
            std::fprintf(f, "CENTER %.9g %.9g %.9g\n", maps->box_center[0], maps->box_center[1], maps->box_center[2]);
            for (size_t i = 0; i < plane; ++i) std::fprintf(f, "%.9g\n", h[i]);
            std::fclose(f);
        }
    });
}

// One AutoGrid .map text file: six header lines (SPACING on the 4th,
// NELEMENTS on the 5th, CENTER on the 6th) then one value per line, x
// fastest (read_vina_map / read_ad4_map, cache.cpp:267-323, ad4cache.cpp:333-389).
static bool read_map_file(const std::string& path, float& spacing, int nvox[3], float center[3],
                          std::vector<float>& vals) {
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    char line[512];
    int ln = 0;
    vals.clear();
    bool ok = true;
    while (std::fgets(line, sizeof line, f)) {
        ++ln;
        if (ln == 4) ok &= std::sscanf(line, "%*s %f", &spacing) == 1;
        else if (ln == 5) ok &= std::sscanf(line, "%*s %d %d %d", &nvox[0], &nvox[1], &nvox[2]) == 3;
        else if (ln == 6) ok &= std::sscanf(line, "%*s %f %f %f", &center[0], &center[1], &center[2]) == 3;
        else if (ln > 6) vals.push_back(std::strtof(line, nullptr));
    }
    std::fclose(f);
    if (!ok) throw Error(UD_ERR_PARSE, "malformed map header in " + path);
    for (int i = 0; i < 3; ++i)
        if (nvox[i] < 2 || nvox[i] % 2 == 1)
            throw Error(UD_ERR_PARSE, "number of voxels (NELEMENTS) must be even and positive in " + path);
    const size_t want = (size_t)(nvox[0] + 1) * (nvox[1] + 1) * (nvox[2] + 1);
    if (vals.size() != want)
        throw Error(UD_ERR_PARSE, path + ": " + std::to_string(vals.size()) + " values, expected " +
                                      std::to_string(want));
    return true;
}

extern "C" int ud_maps_load(int sf, const float* weights, int n_weights, const char* prefix, void* stream,
                            ud_maps* out) {
    return guarded([&] {
        if (!out || !prefix) throw Error(UD_ERR_ARG, "null argument");
        if (sf != UD_SF_VINA && sf != UD_SF_VINARDO && sf != UD_SF_AD4) throw Error(UD_ERR_ARG, "unknown scoring function");
        cudaStream_t s = (cudaStream_t)stream;
        auto m = std::make_unique<ud_maps_s>();
        std::vector<float> w;
        if (weights && n_weights > 0) {
            w.assign(weights, weights + n_weights);
            if (sf != UD_SF_AD4) w.back() = (float)(5 * (double)w.back() / 0.1 - 1);  // as ud_maps_create
        }
        m->sf = Scoring::make(sf == UD_SF_AD4 ? SF_AD42 : sf, w.empty() ? nullptr : w.data(), (int)w.size());
        MapsDesc& d = m->desc;
        std::vector<std::pair<std::string, int>> files;  // (name, type)
        if (sf == UD_SF_AD4) {
            for (int t : default_ad4_types()) files.push_back({ad_kind(t).name, t});
        } else {
            for (int t : default_map_types()) files.push_back({xs_name(t), t});
        }
        std::vector<std::vector<float>> data;
        float spacing0 = 0, center0[3] = {0, 0, 0};
        int nvox0[3] = {0, 0, 0};
        auto take = [&](const std::string& name, int type, bool required) {
            float sp, c[3];
            int nv[3];
            std::vector<float> v;
            const std::string path = std::string(prefix) + "." + name + ".map";
            if (!read_map_file(path, sp, nv, c, v)) {
                if (required) throw Error(UD_ERR_ARG, "missing map file " + path);
                return;
            }
            if (data.empty()) {
                spacing0 = sp;
                for (int i = 0; i < 3; ++i) {
                    nvox0[i] = nv[i];
                    center0[i] = c[i];
                }
            } else if (sp != spacing0 || nv[0] != nvox0[0] || nv[1] != nvox0[1] || nv[2] != nvox0[2] ||
                       c[0] != center0[0] || c[1] != center0[1] || c[2] != center0[2]) {
                throw Error(UD_ERR_ARG, "map " + path + " has a different grid than the others");
            }
            data.push_back(std::move(v));
            if (type >= 0) m->slot_types.push_back(type);
        };
        for (auto& f : files) take(f.first, f.second, false);
        if (m->slot_types.empty()) throw Error(UD_ERR_ARG, std::string("no *.map files with prefix ") + prefix);
        std::fill(d.slot_of_xs, d.slot_of_xs + 36, (int8_t)-1);
        for (size_t k = 0; k < m->slot_types.size(); ++k) d.slot_of_xs[m->slot_types[k]] = (int8_t)k;
        if (sf == UD_SF_AD4) {
            d.ad4 = 1;
            d.e_slot = (int)m->slot_types.size();
            d.d_slot = d.e_slot + 1;
            take("e", -1, true);
            take("d", -1, true);
        }
        d.n_maps = (int)data.size();
        for (int i = 0; i < 3; ++i) {  // grid frame of the map reader (read_ad4_map, ad4cache.cpp:365-376)
            const float halfspan = (float)((double)(nvox0[i] * spacing0) / 2.0);
            const float begin = center0[i] - halfspan, end = center0[i] + halfspan;
            d.dims[i] = nvox0[i] + 1;
            d.init[i] = begin;
            d.corner2[i] = end;
            d.dim_m1[i] = (float)nvox0[i];
            d.factor[i] = d.dim_m1[i] / (end - begin);
            d.factor_inv[i] = 1 / d.factor[i];
        }
        d.slope = 1e6f;
        for (int i = 0; i < 3; ++i) m->box_center[i] = center0[i];
        m->box_spacing = spacing0;
        const PairTable& tab = *cached_table(m->sf);
        m->n_bins = tab.n;
        m->factor = tab.factor;
        m->cutoff2 = m->sf.cutoff * m->sf.cutoff;
        {
            std::vector<float> s4(tab.smooth.size() * 2, 0.0f);
            pack_smooth4(tab, s4.data());
            m->smooth.upload(s4.data(), s4.size(), s);
        }
        m->fast.alloc(round4(tab.fast.size()));
        m->fast.upload(tab.fast.data(), tab.fast.size(), s);
        const size_t plane = (size_t)d.dims[0] * d.dims[1] * d.dims[2];
        std::vector<float> all(round4(plane * d.n_maps), 0.0f);
        for (int k = 0; k < d.n_maps; ++k) std::copy(data[k].begin(), data[k].end(), all.begin() + plane * k);
        m->maps.upload(all.data(), all.size(), s);
        refresh_xpairs(m.get(), s);
        cuda_check(cudaStreamSynchronize(s), "maps upload");
        m->loaded = true;
        *out = m.release();
    });
}

extern "C" int ud_maps_info(ud_maps maps, int dims[3], float init[3], float factor[3], int* n_maps) {
    return guarded([&] {
        if (!maps) throw Error(UD_ERR_ARG, "null maps");
        for (int i = 0; i < 3; ++i) {
            if (dims) dims[i] = maps->desc.dims[i];
            if (init) init[i] = maps->desc.init[i];
            if (factor) factor[i] = maps->desc.factor[i];
        }
        if (n_maps) *n_maps = maps->desc.n_maps;
    });
}

extern "C" int ud_maps_read(ud_maps maps, int xs, float* out, size_t n) {
    return guarded([&] {
        if (!maps || !out || xs < 0) throw Error(UD_ERR_ARG, "invalid argument");
        int slot = -1;
        if (maps->desc.ad4) {  // AD type, AD_SIZE = electrostatic, AD_SIZE + 1 = desolvation
            if (xs == AD_SIZE) slot = maps->desc.e_slot;
            else if (xs == AD_SIZE + 1) slot = maps->desc.d_slot;
            else if (xs < AD_SIZE) slot = maps->desc.slot_of_xs[xs];
            if (slot < 0) throw Error(UD_ERR_ARG, "no AD4 map for type " + std::to_string(xs));
        } else {
            if (xs >= XS_SIZE) throw Error(UD_ERR_ARG, "invalid argument");
            slot = maps->desc.slot_of_xs[xs];
            if (slot < 0) throw Error(UD_ERR_ARG, std::string("no map for type ") + xs_name(xs));
        }
        const size_t plane = (size_t)maps->desc.dims[0] * maps->desc.dims[1] * maps->desc.dims[2];
        if (n < plane) throw Error(UD_ERR_CAPACITY, "output buffer too small");
        cuda_check(cudaMemcpy(out, maps->maps.p + plane * slot, plane * sizeof(float), cudaMemcpyDeviceToHost),
                   "map D2H");
    });
}

extern "C" int ud_maps_destroy(ud_maps maps) {
    delete maps;
    return UD_OK;
}

// ---------------------------------------------------------------- ligands

static int ligand_local_steps(const Ligand& L) { return (25 + (int)L.atoms.size()) / 3; }

// A ligand beyond the search's limits is refused when it is parsed, so that a
// screen skips it alone (parse_ligand_from_file_no_failure refuses more than
// MAX_NUM_OF_LIG_TORSION torsions and MAX_NUM_OF_ATOMS atoms the same way,
// parse_pdbqt.cpp:1107-1120; the atom limit here is 256, the reference's 150).
static Ligand within_limits(Ligand L) {
    if (L.n_torsions() > kMaxLigTorsions)
        throw Error(UD_ERR_CAPACITY, "ligand exceeds max torsion counts: " + std::to_string(L.n_torsions()) +
                                         " > " + std::to_string(kMaxLigTorsions));
    if ((int)L.atoms.size() > kMaxLigAtoms)
        throw Error(UD_ERR_CAPACITY, "ligand exceeds max atom counts: " + std::to_string(L.atoms.size()) + " > " +
                                         std::to_string(kMaxLigAtoms));
    return L;
}

extern "C" int ud_ligand_parse(const char* text, size_t len, ud_ligand* out) {
    return guarded([&] {
        if (!text || !out) throw Error(UD_ERR_ARG, "null argument");
        auto h = std::make_unique<ud_ligand_s>();
        h->lig = within_limits(parse_ligand(std::string(text, len)));
        *out = h.release();
    });
}

extern "C" int ud_ligand_parse_sdf(const char* sdf, size_t len, int keep_h, ud_ligand* out) {
    return guarded([&] {
        if (!sdf || !out) throw Error(UD_ERR_ARG, "null argument");
        auto h = std::make_unique<ud_ligand_s>();
        h->lig = within_limits(parse_ligand_sdf(std::string(sdf, len), keep_h != 0));
        *out = h.release();
    });
}

extern "C" int ud_ligand_parse_many(const char* const* texts, const size_t* lens, int n, int threads,
                                    ud_ligand* out, int* status) {
    return guarded([&] {
        if (n < 0 || (n > 0 && (!texts || !lens || !out))) throw Error(UD_ERR_ARG, "invalid arguments");
        for (int i = 0; i < n; ++i) out[i] = nullptr;
        std::atomic<int> next{0}, failed{0};
        const int nt = std::max(1, std::min(threads > 0 ? threads : (int)std::thread::hardware_concurrency(), n));
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t)
            pool.emplace_back([&] {
                for (int i; (i = next.fetch_add(1)) < n;) {
                    int code = UD_OK;
                    try {
                        if (!texts[i]) throw Error(UD_ERR_ARG, "null text");
                        auto h = std::make_unique<ud_ligand_s>();
                        h->lig = within_limits(parse_ligand(std::string(texts[i], lens[i])));
                        out[i] = h.release();
                    } catch (const Error& e) {
                        code = e.code;
                    } catch (const std::exception&) {
                        code = UD_ERR_PARSE;
                    }
                    if (status) status[i] = code;
                    if (code != UD_OK) failed.fetch_add(1);
                }
            });
        for (auto& th : pool) th.join();
        if (failed.load() > 0 && !status)
            throw Error(UD_ERR_PARSE, std::to_string(failed.load()) + " of " + std::to_string(n) + " ligands failed to parse");
    });
}

extern "C" int ud_ligand_write(ud_ligand lig, const float* pose, char* buf, size_t cap, size_t* len) {
    return guarded([&] {
        if (!lig || !pose) throw Error(UD_ERR_ARG, "null argument");
        const std::string s = write_structure(lig->lig, pose);
        if (len) *len = s.size();
        if (buf && cap > 0) {
            size_t n = std::min(cap - 1, s.size());
            std::memcpy(buf, s.data(), n);
            buf[n] = 0;
        }
    });
}

extern "C" int ud_ligand_counts(ud_ligand lig, int counts[8]) {
    return guarded([&] {
        if (!lig || !counts) throw Error(UD_ERR_ARG, "null argument");
        const Ligand& L = lig->lig;
        counts[0] = (int)L.atoms.size();
        counts[1] = L.n_heavy();
        counts[2] = L.n_torsions();
        counts[3] = (int)L.nodes.size();
        counts[4] = (int)L.pairs.size();
        counts[5] = L.torsdof;
        counts[6] = (int)L.glue_pairs.size();
        counts[7] = ligand_local_steps(L);
    });
}

extern "C" int ud_ligand_export(ud_ligand lig, float* lab_xyz, float* local_xyz, int* xs, int* ad,
                                int* el, float* charge, int* atom_node, int* node_parent, int* node_begin,
                                int* node_end, float* node_rel, int* pair_a, int* pair_b) {
    return guarded([&] {
        if (!lig) throw Error(UD_ERR_ARG, "null ligand");
        const Ligand& L = lig->lig;
        for (size_t i = 0; i < L.atoms.size(); ++i) {
            const Atom& a = L.atoms[i];
            for (int k = 0; k < 3; ++k) {
                if (lab_xyz) lab_xyz[3 * i + k] = a.lab[k];
                if (local_xyz) local_xyz[3 * i + k] = a.local[k];
            }
            if (xs) xs[i] = a.xs;
            if (ad) ad[i] = a.ad;
            if (el) el[i] = a.el;
            if (charge) charge[i] = a.charge;
            if (atom_node) atom_node[i] = a.node;
        }
        for (size_t n = 0; n < L.nodes.size(); ++n) {
            const Node& nd = L.nodes[n];
            if (node_parent) node_parent[n] = nd.parent;
            if (node_begin) node_begin[n] = nd.begin;
            if (node_end) node_end[n] = nd.end;
            if (node_rel)
                for (int k = 0; k < 3; ++k) {
                    node_rel[6 * n + k] = nd.rel_origin[k];
                    node_rel[6 * n + 3 + k] = nd.rel_axis[k];
                }
        }
        for (size_t p = 0; p < L.pairs.size(); ++p) {
            if (pair_a) pair_a[p] = L.pairs[p].a;
            if (pair_b) pair_b[p] = L.pairs[p].b;
        }
    });
}

extern "C" int ud_ligand_initial_pose(ud_ligand lig, float* pose) {
    return guarded([&] {
        if (!lig || !pose) throw Error(UD_ERR_ARG, "null argument");
        const Ligand& L = lig->lig;
        for (int k = 0; k < 3; ++k) pose[k] = L.nodes[0].origin0[k];
        pose[3] = 1; pose[4] = 0; pose[5] = 0; pose[6] = 0;
        for (int t = 0; t < L.n_torsions(); ++t) pose[7 + t] = 0;
    });
}

extern "C" int ud_ligand_coords(ud_ligand lig, const float* pose, float* xyz) {
    return guarded([&] {
        if (!lig || !pose || !xyz) throw Error(UD_ERR_ARG, "null argument");
        ligand_coords(lig->lig, pose, xyz);
    });
}

extern "C" int ud_ligand_conf_indep(ud_ligand lig, float out[7]) {
    return guarded([&] {
        if (!lig || !out) throw Error(UD_ERR_ARG, "null argument");
        auto v = lig->lig.conf_indep_inputs();
        for (int i = 0; i < 7; ++i) out[i] = v[i];
    });
}

extern "C" int ud_ligand_destroy(ud_ligand lig) {
    delete lig;
    return UD_OK;
}

// ---------------------------------------------------------------- batches

// Index into `pairs` of every slot of the conflict-free 32-slot groups, -1 for
// padding: each group is kPairPasses lane ranges of kPairPassWidth slots, and
// no atom occurs twice within a range (the kernel adds one range's forces at a
// time).  Ranges are filled greedily in pair order.
static std::vector<int> pair_group_slots(const Ligand& L, const std::vector<Pair>& pairs) {
    std::vector<int> out;
    std::vector<char> used(pairs.size(), 0);
    std::vector<int> stamp(L.atoms.size(), -1);
    size_t left = pairs.size(), start = 0;
    int range_id = 0;
    while (left > 0) {
        for (int r = 0; r < kPairPasses; ++r, ++range_id) {
            int filled = 0;
            for (size_t k = start; k < pairs.size() && filled < kPairPassWidth; ++k) {
                if (used[k]) continue;
                const Pair& p = pairs[k];
                if (stamp[p.a] == range_id || stamp[p.b] == range_id) continue;
                stamp[p.a] = stamp[p.b] = range_id;
                used[k] = 1;
                --left;
                ++filled;
                out.push_back((int)k);
            }
            while (start < pairs.size() && used[start]) ++start;
            while (filled++ < kPairPassWidth) out.push_back(-1);
        }
    }
    return out;
}

// Host records of the device topology of `ligs` against `maps`: LigDesc,
// atoms, nodes, pair words, grid-atom list (and AD4 charges / pair
// coefficients), with every LigDesc offset counted from the given bases (0
// for a batch of its own; a streaming screen appends slot after slot to one
// arena), and the work order of the persistent search (most expensive ligands
// first, BFGS steps x (atoms + pairs) as the cost proxy) as lig_base + index.
struct TopologyPack {
    std::vector<LigDesc> desc;
    std::vector<AtomRec> atoms;
    std::vector<NodeRec> nodes;
    std::vector<uint32_t> pairs;
    std::vector<uint32_t> grid_list;
    std::vector<float> charges, coef;  // AD4 only
    std::vector<int> order;
    int max_atoms = 0, max_tors = 0;
};

static void pack_topology(const ud_maps_s* maps, const std::vector<const Ligand*>& ligs, int lig_base,
                          size_t atom_base, size_t node_base, size_t pair_base, size_t grid_base, TopologyPack& tp) {
        const int n = (int)ligs.size();
        tp = TopologyPack{};
        auto& atoms = tp.atoms;
        auto& nodes = tp.nodes;
        auto& pairs = tp.pairs;
        auto& grid_list = tp.grid_list;
        auto& charges = tp.charges;
        auto& coef = tp.coef;
        for (int i = 0; i < n; ++i) {
            const Ligand& L = *ligs[i];
            if ((int)L.atoms.size() > kMaxLigAtoms)
                throw Error(UD_ERR_CAPACITY, "ligand " + std::to_string(i) + " has more than 256 atoms");
            if (L.n_torsions() > kMaxLigTorsions)
                throw Error(UD_ERR_CAPACITY, "ligand " + std::to_string(i) + " has more than 48 torsions");
            LigDesc d{};
            d.atom_off = (int)(atom_base + atoms.size());
            d.n_atoms = (int)L.atoms.size();
            d.node_off = (int)(node_base + nodes.size());
            d.n_nodes = (int)L.nodes.size();
            d.pair_off = (int)(pair_base + pairs.size());
            d.n_heavy = L.n_heavy();
            d.local_steps = ligand_local_steps(L);
            std::vector<int> depth(L.nodes.size(), 0);
            for (size_t k = 1; k < L.nodes.size(); ++k) depth[k] = depth[L.nodes[k].parent] + 1;
            d.max_depth = *std::max_element(depth.begin(), depth.end());
            std::vector<int> subtree_end(L.nodes.size());
            for (size_t k = 0; k < L.nodes.size(); ++k) subtree_end[k] = (int)k + 1;
            for (size_t k = L.nodes.size(); k-- > 1;)  // children have larger DFS indices
                subtree_end[L.nodes[k].parent] = std::max(subtree_end[L.nodes[k].parent], subtree_end[k]);
            for (size_t k = 0; k < L.nodes.size(); ++k) {
                const Node& nd = L.nodes[k];
                NodeRec r{};
                for (int q = 0; q < 3; ++q) {
                    r.rel_origin[q] = nd.rel_origin[q];
                    r.rel_axis[q] = nd.rel_axis[q];
                }
                r.parent = nd.parent < 0 ? 0 : nd.parent;
                r.depth = depth[k];
                // a subtree's atoms are contiguous in DFS order: [own begin, last descendant's end)
                r.atoms = nd.begin | (L.nodes[subtree_end[k] - 1].end << 16);
                r.subtree_end = subtree_end[k];
                nodes.push_back(r);
            }
            d.grid_off = (int)(grid_base + grid_list.size());
            const size_t atom0 = atoms.size(), grid0 = grid_list.size(), pair0 = pairs.size();
            const bool ad4 = maps->desc.ad4 != 0;
            for (const Atom& a : L.atoms) {
                AtomRec r;
                r.x = a.local[0];
                r.y = a.local[1];
                r.z = a.local[2];
                int g, slot;
                if (ad4) {  // every AD-typed atom but glue atoms; CG carbons read the C map (ad4cache.cpp:227-269)
                    g = (a.ad < AD_SIZE && (a.ad < AD_G0 || a.ad > AD_G3)) ? a.ad : -1;
                    if (g >= AD_CG0 && g <= AD_CG3) g = AD_C;
                    slot = (g >= 0) ? maps->desc.slot_of_xs[g] : -1;
                    if (g >= 0 && slot < 0)
                        throw Error(UD_ERR_ARG, std::string("no AD4 map for ligand atom type ") + ad_kind(g).name);
                    charges.push_back(a.charge);
                } else {
                    g = (a.xs < XS_SIZE) ? xs_grid_type(a.xs) : -1;
                    slot = (g >= 0) ? maps->desc.slot_of_xs[g] : -1;
                    if (g >= 0 && slot < 0)
                        throw Error(UD_ERR_ARG, std::string("no grid map for ligand atom type ") + xs_name(g));
                }
                int heavy = (a.el != EL_H) ? 1 : 0;
                int xsp = (a.xs < XS_SIZE) ? a.xs + 1 : 0;
                r.packed = a.node | ((slot + 1) << 8) | (heavy << 16) | (xsp << 24);
                if (slot >= 0) grid_list.push_back((uint32_t)(atoms.size() - atom0) | ((uint32_t)slot << 8));
                atoms.push_back(r);
            }
            d.n_grid = (int)(grid_list.size() - grid0);
            const std::vector<Pair>& plist = ad4 ? L.pairs_ad : L.pairs;
            for (int k : pair_group_slots(L, plist)) {
                if (k < 0) {
                    pairs.push_back(kPairPad);
                    if (ad4) {
                        coef.push_back(0.0f);
                        coef.push_back(0.0f);
                    }
                    continue;
                }
                const Pair& p = plist[k];
                pairs.push_back((uint32_t)p.a | ((uint32_t)p.b << 8) | ((uint32_t)p.tp << 16));
                if (ad4) {  // per-pair scales of the shared electrostatic and desolvation rows
                    const Atom &x = L.atoms[p.a], &y = L.atoms[p.b];
                    coef.push_back(x.charge * y.charge);
                    coef.push_back(std::fabs(x.charge) * ad4_volume(y.ad) + std::fabs(y.charge) * ad4_volume(x.ad));
                }
            }
            d.n_pairs = (int)(pairs.size() - pair0);
            tp.desc.push_back(d);
            tp.max_atoms = std::max(tp.max_atoms, d.n_atoms);
            tp.max_tors = std::max(tp.max_tors, d.n_nodes - 1);
        }
        std::vector<int> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            long long cx = (long long)tp.desc[x].local_steps * (tp.desc[x].n_atoms + tp.desc[x].n_pairs);
            long long cy = (long long)tp.desc[y].local_steps * (tp.desc[y].n_atoms + tp.desc[y].n_pairs);
            return cx > cy;
        });
        for (int& o : order) o += lig_base;
        tp.order = std::move(order);
}

// Topology of `ligs` into the batch's device arrays (grown, never shrunk, so a
// batch reused for the next ligands allocates nothing once it has seen the
// largest batch).  The work order is uploaded with the topology, so that a
// search launch does no host-to-device copy (a copy from pageable memory would
// wait for the stream's prior work).
static void fill_batch(ud_batch_s* b, const std::vector<const Ligand*>& ligs, cudaStream_t s) {
        const int n = (int)ligs.size();
        TopologyPack tp;
        pack_topology(b->maps, ligs, 0, 0, 0, 0, 0, tp);
        b->ligs = ligs;
        b->desc = tp.desc;
        b->max_atoms = tp.max_atoms;
        b->max_tors = tp.max_tors;
        b->d_desc.upload(b->desc.data(), b->desc.size(), s);
        b->d_atoms.upload(tp.atoms.data(), tp.atoms.size(), s);
        b->d_nodes.upload(tp.nodes.data(), tp.nodes.size(), s);
        b->d_pairs.upload(tp.pairs.data(), tp.pairs.size(), s);
        b->d_grid.upload(tp.grid_list.data(), tp.grid_list.size(), s);
        b->upload_bytes = b->desc.size() * sizeof(LigDesc) + tp.atoms.size() * sizeof(AtomRec) +
                          tp.nodes.size() * sizeof(NodeRec) + (tp.pairs.size() + tp.grid_list.size()) * 4 +
                          (size_t)n * sizeof(int);
        if (b->maps->desc.ad4) {
            b->d_charge.upload(tp.charges.data(), tp.charges.size(), s);
            b->d_pair_coef.upload(tp.coef.data(), tp.coef.size(), s);
            b->upload_bytes += (tp.charges.size() + tp.coef.size()) * sizeof(float);
        }
        b->d_order.upload(tp.order.data(), tp.order.size(), s);
        cuda_check(cudaStreamSynchronize(s), "batch upload");
}

static std::unique_ptr<ud_batch_s> build_batch(ud_maps maps, const std::vector<const Ligand*>& ligs,
                                               cudaStream_t s) {
    auto b = std::make_unique<ud_batch_s>();
    b->maps = maps;
    fill_batch(b.get(), ligs, s);
    return b;
}

// Bytes of one DevBuf allocation of `count` elements of `size` bytes (its
// quarter of headroom included).
static size_t devbuf_bytes(size_t count, size_t size) { return std::max<size_t>(count + count / 4, 1) * size; }

extern "C" int ud_batch_device_bytes(const ud_ligand* ligs, int n, int sf, const ud_search_params* params,
                                     size_t* bytes) {
    return guarded([&] {
        if (!bytes || !params || n < 0 || (n > 0 && !ligs)) throw Error(UD_ERR_ARG, "invalid arguments");
        if (sf != UD_SF_VINA && sf != UD_SF_VINARDO && sf != UD_SF_AD4) throw Error(UD_ERR_ARG, "unknown scoring");
        const bool ad4 = sf == UD_SF_AD4;
        size_t atoms = 0, nodes = 0, slots = 0;
        int max_atoms = 0, max_tors = 0;
        for (int i = 0; i < n; ++i) {
            if (!ligs[i]) throw Error(UD_ERR_ARG, "null ligand");
            const Ligand& L = ligs[i]->lig;
            std::atomic<int>& cached = ligs[i]->pair_slots[ad4 ? 1 : 0];
            int ps = cached.load(std::memory_order_relaxed);
            if (ps < 0) {
                ps = (int)pair_group_slots(L, ad4 ? L.pairs_ad : L.pairs).size();
                cached.store(ps, std::memory_order_relaxed);
            }
            atoms += L.atoms.size();
            nodes += L.nodes.size();
            slots += (size_t)ps;
            max_atoms = std::max(max_atoms, (int)L.atoms.size());
            max_tors = std::max(max_tors, L.n_torsions());
        }
        const size_t E = (size_t)std::max(1, params->exhaustiveness), cap = (size_t)std::max(1, params->num_modes);
        const size_t stride = 7 + (size_t)max_tors, chains = (size_t)n * E, mode_slots = (size_t)n * cap;
        size_t b = 0;
        // topology (fill_batch)
        b += devbuf_bytes(n, sizeof(LigDesc)) + devbuf_bytes(atoms, sizeof(AtomRec)) +
             devbuf_bytes(nodes, sizeof(NodeRec)) + devbuf_bytes(slots, sizeof(uint32_t)) +
             devbuf_bytes(atoms, sizeof(uint32_t)) + devbuf_bytes(n, sizeof(int));
        if (ad4) b += devbuf_bytes(atoms, sizeof(float)) + devbuf_bytes(slots, 2 * sizeof(float));
        // search results (search_launch)
        b += devbuf_bytes(chains * stride, sizeof(float)) + devbuf_bytes(chains, sizeof(ChainResult)) +
             devbuf_bytes(1, sizeof(unsigned int));
        // modes (alloc_modes)
        b += devbuf_bytes(mode_slots * 3 * std::max(1, max_atoms), sizeof(float)) + devbuf_bytes(n, sizeof(int)) +
             2 * devbuf_bytes(mode_slots, sizeof(int)) + devbuf_bytes(mode_slots * stride, sizeof(float)) +
             devbuf_bytes(mode_slots * 4, sizeof(float));
        *bytes = b;
    });
}

extern "C" int ud_batch_create(ud_maps maps, const ud_ligand* ligs, int n, void* stream, ud_batch* out) {
    return guarded([&] {
        if (!maps || !out || n < 0 || (n > 0 && !ligs)) throw Error(UD_ERR_ARG, "invalid batch arguments");
        std::vector<const Ligand*> v;
        for (int i = 0; i < n; ++i) {
            if (!ligs[i]) throw Error(UD_ERR_ARG, "null ligand in batch");
            v.push_back(&ligs[i]->lig);
        }
        *out = build_batch(maps, v, (cudaStream_t)stream).release();
    });
}

extern "C" int ud_batch_reset(ud_batch b, const ud_ligand* ligs, int n, void* stream) {
    return guarded([&] {
        if (!b || n < 0 || (n > 0 && !ligs)) throw Error(UD_ERR_ARG, "invalid batch arguments");
        if (b->launched) throw Error(UD_ERR_STATE, "the batch's launched search has not been collected");
        std::vector<const Ligand*> v;
        for (int i = 0; i < n; ++i) {
            if (!ligs[i]) throw Error(UD_ERR_ARG, "null ligand in batch");
            v.push_back(&ligs[i]->lig);
        }
        b->searched = false;
        b->post.clear();
        b->text[0].clear();
        b->text[1].clear();
        b->text_ready[0] = b->text_ready[1] = false;
        b->tuned = false;
        b->lig_bias.clear();
        b->lig_bias_dirty = true;
        fill_batch(b, v, (cudaStream_t)stream);
    });
}

extern "C" int ud_batch_destroy(ud_batch batch) {
    delete batch;
    return UD_OK;
}

// ---------------------------------------------------------------- scoring

static void check_poses(ud_batch b, const int* pose_ligand, int n_poses, int pose_stride) {
    if (!b || n_poses < 0 || !pose_ligand) throw Error(UD_ERR_ARG, "invalid pose arguments");
    if (pose_stride < 7 + b->max_tors) throw Error(UD_ERR_ARG, "pose_stride smaller than 7 + max torsions");
}

extern "C" int ud_score_grad_device(ud_batch b, const int* pose_ligand, const float* poses, int n_poses,
                                    int pose_stride, float v_intra, float v_inter, float* e_out, float* g_out,
                                    int g_stride, void* stream) {
    return guarded([&] {
        if (!b || !poses || !e_out || !g_out || g_stride < 6 + b->max_tors)
            throw Error(UD_ERR_ARG, "invalid score arguments");
        if (pose_stride < 7 + b->max_tors) throw Error(UD_ERR_ARG, "pose_stride too small");
        if (n_poses == 0) return;
        cuda_check(launch_score(b->view(), maps_view(b->maps), tables_view(b->maps), pose_ligand, poses,
                                pose_stride, n_poses, v_intra, v_inter, e_out, g_out, g_stride, nullptr,
                                (cudaStream_t)stream),
                   "score kernel");
    });
}

extern "C" int ud_score_grad(ud_batch b, const int* pose_ligand, const float* poses, int n_poses,
                             int pose_stride, float v_intra, float v_inter, float* e_out, float* g_out,
                             int g_stride, void* stream) {
    return guarded([&] {
        check_poses(b, pose_ligand, n_poses, pose_stride);
        if (!poses || !e_out || !g_out || g_stride < 6 + b->max_tors) throw Error(UD_ERR_ARG, "invalid buffers");
        for (int i = 0; i < n_poses; ++i)
            if (pose_ligand[i] < 0 || pose_ligand[i] >= (int)b->desc.size())
                throw Error(UD_ERR_ARG, "pose_ligand out of range");
        if (n_poses == 0) return;
        cudaStream_t s = (cudaStream_t)stream;
        b->d_pose_lig.upload(pose_ligand, n_poses, s);
        b->d_pose.upload(poses, (size_t)n_poses * pose_stride, s);
        b->d_e.alloc(n_poses);
        b->d_g.alloc((size_t)n_poses * g_stride);
        // entries past a pose's 6 + T gradient floats come back as 0
        cuda_check(cudaMemsetAsync(b->d_g.p, 0, (size_t)n_poses * g_stride * sizeof(float), s), "memset");
        cuda_check(launch_score(b->view(), maps_view(b->maps), tables_view(b->maps), b->d_pose_lig.p, b->d_pose.p,
                                pose_stride, n_poses, v_intra, v_inter, b->d_e.p, b->d_g.p, g_stride, nullptr, s),
                   "score kernel");
        cuda_check(cudaMemcpyAsync(e_out, b->d_e.p, n_poses * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaMemcpyAsync(g_out, b->d_g.p, (size_t)n_poses * g_stride * sizeof(float),
                                   cudaMemcpyDeviceToHost, s),
                   "D2H");
        cuda_check(cudaStreamSynchronize(s), "score sync");
    });
}

static void score_poses_device(ud_batch b, const std::vector<int>& lig, const std::vector<float>& poses,
                               int stride, float v, std::vector<float>& out, cudaStream_t s) {
    const int n = (int)lig.size();
    out.assign(2 * (size_t)n, 0.0f);
    if (n == 0) return;
    b->d_pose_lig.upload(lig.data(), n, s);
    b->d_pose.upload(poses.data(), poses.size(), s);
    b->d_score.alloc(2 * (size_t)n);
    cuda_check(launch_score(b->view(), maps_view(b->maps), tables_view(b->maps), b->d_pose_lig.p, b->d_pose.p,
                            stride, n, v, v, nullptr, nullptr, 0, b->d_score.p, s),
               "score kernel");
    cuda_check(cudaMemcpyAsync(out.data(), b->d_score.p, 2 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, s),
               "D2H");
    cuda_check(cudaStreamSynchronize(s), "score sync");
}

extern "C" int ud_score(ud_batch b, const int* pose_ligand, const float* poses, int n_poses, int pose_stride,
                        float v, float* out, void* stream) {
    return guarded([&] {
        check_poses(b, pose_ligand, n_poses, pose_stride);
        if (!poses || !out) throw Error(UD_ERR_ARG, "null buffer");
        for (int i = 0; i < n_poses; ++i)
            if (pose_ligand[i] < 0 || pose_ligand[i] >= (int)b->desc.size())
                throw Error(UD_ERR_ARG, "pose_ligand out of range");
        std::vector<int> l(pose_ligand, pose_ligand + n_poses);
        std::vector<float> p(poses, poses + (size_t)n_poses * pose_stride), o;
        score_poses_device(b, l, p, pose_stride, v, o, (cudaStream_t)stream);
        std::copy(o.begin(), o.end(), out);
    });
}

// Vina::score of fixed poses (vina.cpp:1168-1240) for a rigid receptor: per
// pose {total, ligand-receptor, ligand-flex, flex-receptor, flex-flex intra,
// ligand intra, conf-independent, unbound}; the unbound energy is the pose's
// own intramolecular energy (Vina::score, vina.cpp:1329-1355).
extern "C" int ud_score_terms(ud_batch b, const int* pose_ligand, const float* poses, int n_poses, int pose_stride,
                              float* out, void* stream) {
    return guarded([&] {
        check_poses(b, pose_ligand, n_poses, pose_stride);
        if (!poses || !out) throw Error(UD_ERR_ARG, "null buffer");
        for (int i = 0; i < n_poses; ++i)
            if (pose_ligand[i] < 0 || pose_ligand[i] >= (int)b->desc.size())
                throw Error(UD_ERR_ARG, "pose_ligand out of range");
        std::vector<int> l(pose_ligand, pose_ligand + n_poses);
        std::vector<float> p(poses, poses + (size_t)n_poses * pose_stride), sc;
        score_poses_device(b, l, p, pose_stride, 1000.0f, sc, (cudaStream_t)stream);
        const Scoring& sf = b->maps->sf;
        const bool ad4 = sf.choice == SF_AD42;
        for (int i = 0; i < n_poses; ++i) {
            const Ligand& L = *b->ligs[pose_ligand[i]];
            const float grid = sc[2 * i], intra = sc[2 * i + 1];
            const float num_tors = L.conf_indep_inputs()[0];
            // AD4 adds the torsional term to the inter energy alone and reports
            // -intra as the unbound energy (vina.cpp:1207-1237)
            const float total = ad4 ? grid + sf.conf_independent(0.0f, num_tors, (float)L.torsdof)
                                    : sf.conf_independent(grid + intra - intra, num_tors, (float)L.torsdof);
            float* o = out + 8 * (size_t)i;
            o[0] = total;
            o[1] = grid;
            o[2] = 0.0f;
            o[3] = 0.0f;
            o[4] = 0.0f;
            o[5] = intra;
            o[6] = total - grid;
            o[7] = ad4 ? -intra : intra;
        }
    });
}

// ---------------------------------------------------------------- bias wells

static BiasRec bias_rec(const BiasElement& e) {
    BiasRec r{};
    r.x = e.xyz[0];
    r.y = e.xyz[1];
    r.z = e.xyz[2];
    r.vset = e.vset;
    r.r = e.r;
    bias_atom_multiplicity(e, r.mult);
    return r;
}

extern "C" int ud_maps_add_bias(ud_maps m, const char* text, size_t len, void* stream) {
    return guarded([&] {
        if (!m || !text) throw Error(UD_ERR_ARG, "null argument");
        if (m->terms_built)
            throw Error(UD_ERR_STATE, "add bias wells before the maps' term decomposition is first used");
        cudaStream_t s = (cudaStream_t)stream;
        const std::vector<BiasElement> wells = parse_bias(std::string(text, len));
        if (m->desc.ad4) {
            // AutoDock 4.2: the wells go into the maps only (ad4cache::set_bias);
            // receptor-atom scoring is for Vina / Vinardo maps
            std::vector<BiasMapRec> recs;
            for (const BiasElement& e : wells) {
                BiasMapRec r{};
                r.x = e.xyz[0];
                r.y = e.xyz[1];
                r.z = e.xyz[2];
                r.vset = e.vset;
                r.r = e.r;
                const uint64_t types = bias_ad4_map_types(e);
                auto set = [&](int k) {
                    if (k < 32) r.slots_lo |= 1u << k;
                    else r.slots_hi |= 1u << (k - 32);
                };
                for (size_t k = 0; k < m->slot_types.size(); ++k)
                    if ((types >> m->slot_types[k]) & 1u) set((int)k);
                if (types == ~(uint64_t)0) {  // every map: the electrostatic and desolvation maps too
                    set(m->desc.e_slot);
                    set(m->desc.d_slot);
                }
                recs.push_back(r);
            }
            DevBuf<BiasMapRec> d;
            d.upload(recs.data(), recs.size(), s);
            cuda_check(launch_bias_maps(d.p, (int)recs.size(), m->desc, m->maps.p, s), "bias maps kernel");
            refresh_xpairs(m, s);
            cuda_check(cudaStreamSynchronize(s), "bias maps");
            m->bias.insert(m->bias.end(), wells.begin(), wells.end());
            return;
        }
        std::vector<BiasMapRec> recs;
        for (const BiasElement& e : wells) {
            BiasMapRec r{};
            r.x = e.xyz[0];
            r.y = e.xyz[1];
            r.z = e.xyz[2];
            r.vset = e.vset;
            r.r = e.r;
            const uint64_t types = bias_map_types(e);
            for (size_t k = 0; k < m->slot_types.size(); ++k)
                if ((types >> m->slot_types[k]) & 1u) {
                    if (k < 32) r.slots_lo |= 1u << k;
                    else r.slots_hi |= 1u << (k - 32);
                }
            recs.push_back(r);
        }
        DevBuf<BiasMapRec> d;
        d.upload(recs.data(), recs.size(), s);
        cuda_check(launch_bias_maps(d.p, (int)recs.size(), m->desc, m->maps.p, s), "bias maps kernel");
        refresh_xpairs(m, s);
        cuda_check(cudaStreamSynchronize(s), "bias maps");
        m->bias.insert(m->bias.end(), wells.begin(), wells.end());
        std::vector<BiasRec> all;
        for (const BiasElement& e : m->bias) all.push_back(bias_rec(e));
        m->d_bias.upload(all.data(), all.size(), s);
        cuda_check(cudaStreamSynchronize(s), "bias upload");
        m->rc.bias = m->d_bias.p;
        m->rc.n_bias = (int)all.size();
    });
}

extern "C" int ud_batch_set_bias(ud_batch b, int lig, const char* text, size_t len) {
    return guarded([&] {
        if (!b || (len > 0 && !text)) throw Error(UD_ERR_ARG, "null argument");
        if (lig < 0 || lig >= (int)b->ligs.size()) throw Error(UD_ERR_ARG, "ligand out of range");
        if (b->maps->desc.ad4) throw Error(UD_ERR_STATE, "bias wells with AutoDock 4.2 maps are not supported by this engine");
        b->lig_bias.resize(b->ligs.size());
        b->lig_bias[lig].clear();
        for (const BiasElement& e : parse_bias(std::string(text ? text : "", len))) b->lig_bias[lig].push_back(bias_rec(e));
        if (b->lig_bias[lig].size() > 0xFFFF) throw Error(UD_ERR_CAPACITY, "too many bias wells for one ligand");
        b->lig_bias_dirty = true;
    });
}

// Per-ligand wells to the device before a receptor-atom launch that needs them.
static void upload_lig_bias(ud_batch b, cudaStream_t s) {
    if (!b->lig_bias_dirty) return;
    std::vector<BiasRec> all;
    std::vector<int> span(b->ligs.size(), 0);
    for (size_t l = 0; l < b->lig_bias.size() && l < b->ligs.size(); ++l) {
        if (b->lig_bias[l].empty()) continue;
        if (all.size() > 0xFFFF) throw Error(UD_ERR_CAPACITY, "too many bias wells in one batch");
        span[l] = (int)all.size() | ((int)b->lig_bias[l].size() << 16);
        all.insert(all.end(), b->lig_bias[l].begin(), b->lig_bias[l].end());
    }
    b->d_lig_bias.upload(all.data(), all.size(), s);
    b->d_lig_bias_span.upload(span.data(), span.size(), s);
    cuda_check(cudaStreamSynchronize(s), "bias upload");
    b->lig_bias_dirty = false;
}

// The receptor view of a batch: the maps' receptor and wells, the batch's per-ligand wells.
static DeviceReceptorView receptor_view(ud_batch b) {
    DeviceReceptorView r = b->maps->rc;
    const bool any = !b->lig_bias.empty();
    r.lig_bias = any ? b->d_lig_bias.p : nullptr;
    r.lig_bias_span = any ? b->d_lig_bias_span.p : nullptr;
    return r;
}

// ---------------------------------------------------------------- adjoint

// Unweighted per-term maps and tables of the maps' scoring function: the
// same construction as the weighted ones (ud_maps_create) with one term at
// weight 1.  Maps and tables are linear in the term weights, so a weighted
// map or table is the weight-sum of these (up to FP32 rounding).
static size_t term_map_block(const ud_maps_s* m) {
    const size_t plane = (size_t)m->desc.dims[0] * m->desc.dims[1] * m->desc.dims[2];
    return round4(plane * std::max(1, m->desc.n_maps));
}
static size_t table_rows(const ud_maps_s* m) {
    return m->desc.ad4 ? (size_t)kAd4Rows : (size_t)XS_SIZE * (XS_SIZE + 1) / 2;
}

static void ensure_terms(ud_maps_s* m, cudaStream_t s) {
    if (m->terms_built) return;
    if (m->loaded)
        throw Error(UD_ERR_STATE, "maps read from files have no per-term decomposition (build them from the receptor)");
    if (!m->bias.empty())
        throw Error(UD_ERR_STATE, "maps with bias wells have no per-term decomposition (the wells are no weighted term)");
    const MapsDesc& d = m->desc;
    const int nt = m->sf.n_terms;
    const int nslot = d.n_maps, nslot_pad = std::max(4, (nslot + 3) & ~3);
    const size_t mblock = term_map_block(m);
    const size_t rblock = table_rows(m) * m->n_bins * 4;
    const size_t fblock = round4(table_rows(m) * m->n_bins);
    m->term_maps.alloc((size_t)nt * mblock);
    m->term_rows.alloc((size_t)nt * rblock);
    m->term_fast.alloc((size_t)nt * fblock);
    cuda_check(cudaMemsetAsync(m->term_maps.p, 0, (size_t)nt * mblock * sizeof(float), s), "memset");
    cuda_check(cudaMemsetAsync(m->term_fast.p, 0, (size_t)nt * fblock * sizeof(float), s), "memset");
    DevBuf<float> d_rec;
    DevBuf<int> d_ad;
    if (d.ad4) {
        d_rec.upload(m->rec_xyzq.data(), m->rec_xyzq.size(), s);
        d_ad.upload(m->rec_ad.data(), m->rec_ad.size(), s);
    } else {
        d_rec.upload(m->rec_xyzt.data(), m->rec_xyzt.size(), s);
    }
    DevBuf<float> d_fastT;
    std::vector<float> rows(rblock), fastT(d.ad4 ? 0 : (size_t)XS_SIZE * m->n_bins * nslot_pad, 0.0f);
    for (int t = 0; t < nt; ++t) {
        const PairTable& tab = *cached_table(m->sf, t);
        if (tab.n != m->n_bins) throw Error(UD_ERR_ARG, "term table size mismatch");
        pack_smooth4(tab, rows.data());
        cuda_check(cudaMemcpyAsync(m->term_rows.p + (size_t)t * rblock, rows.data(), rblock * sizeof(float),
                                   cudaMemcpyHostToDevice, s),
                   "H2D");
        cuda_check(cudaMemcpyAsync(m->term_fast.p + (size_t)t * fblock, tab.fast.data(), tab.fast.size() * sizeof(float),
                                   cudaMemcpyHostToDevice, s),
                   "H2D");
        if (d.ad4) {
            Ad4MapSpec spec = ad4_spec(m, t);
            cuda_check(launch_maps_ad4(d_rec.p, d_ad.p, (int)m->rec_ad.size(), ad4_params(), spec, d,
                                       m->term_maps.p + (size_t)t * mblock, s),
                       "AD4 term maps kernel");
        } else {
            pack_fastT(tab, m->slot_types, nslot_pad, fastT.data());
            d_fastT.upload(fastT.data(), fastT.size(), s);
            if (nslot > 0)
                cuda_check(launch_maps(d_rec.p, (int)(m->rec_xyzt.size() / 4), d_fastT.p, tab.n, nslot, nslot_pad,
                                       tab.factor, m->cutoff2, d, m->term_maps.p + (size_t)t * mblock, s),
                           "term maps kernel");
        }
        // host rows / fastT and the table are reused or freed next round: wait for their copies
        cuda_check(cudaStreamSynchronize(s), "term maps sync");
    }
    m->terms_built = true;
}

static DeviceTermsView terms_view(const ud_maps_s* m) {
    return DeviceTermsView{m->term_maps.p, m->term_rows.p, m->sf.n_terms, (long long)term_map_block(m),
                           (long long)(table_rows(m) * m->n_bins)};
}

extern "C" int ud_maps_term_count(ud_maps maps, int* n_terms) {
    return guarded([&] {
        if (!maps || !n_terms) throw Error(UD_ERR_ARG, "null argument");
        *n_terms = maps->sf.n_terms;
    });
}

extern "C" int ud_maps_get_weights(ud_maps maps, float* w, int n) {
    return guarded([&] {
        if (!maps || !w || n < maps->sf.n_terms) throw Error(UD_ERR_ARG, "invalid weights buffer");
        for (int t = 0; t < maps->sf.n_terms; ++t) w[t] = maps->sf.weights[t];
    });
}

extern "C" int ud_maps_set_weights(ud_maps maps, const float* w, int n, void* stream) {
    return guarded([&] {
        if (!maps || !w || n != maps->sf.n_terms) throw Error(UD_ERR_ARG, "expected one weight per scoring term");
        for (int t = 0; t < n; ++t)
            if (!std::isfinite(w[t])) throw Error(UD_ERR_ARG, "weights must be finite");
        cudaStream_t s = (cudaStream_t)stream;
        ensure_terms(maps, s);
        const size_t rblock = table_rows(maps) * maps->n_bins * 4;
        const size_t fblock = round4(table_rows(maps) * maps->n_bins);
        cuda_check(launch_combine_terms(maps->term_maps.p, (long long)term_map_block(maps), n, w, maps->maps.p, s),
                   "combine maps");
        refresh_xpairs(maps, s);
        cuda_check(launch_combine_terms(maps->term_rows.p, (long long)rblock, n, w, maps->smooth.p, s), "combine rows");
        cuda_check(launch_combine_terms(maps->term_fast.p, (long long)fblock, n, w, maps->fast.p, s), "combine fast");
        for (int t = 0; t < n; ++t) maps->sf.weights[t] = w[t];
    });
}

extern "C" int ud_score_adjoint_device(ud_batch b, const int* pose_ligand, const float* poses, int n_poses,
                                       int pose_stride, float v_intra, float v_inter, int flags, float* e_out,
                                       float* g_out, int g_stride, float* dw_out, int dw_stride, void* stream) {
    return guarded([&] {
        if (!b || n_poses < 0 || (n_poses > 0 && (!pose_ligand || !poses || !e_out)))
            throw Error(UD_ERR_ARG, "invalid adjoint arguments");
        if (pose_stride < 7 + b->max_tors) throw Error(UD_ERR_ARG, "pose_stride smaller than 7 + max torsions");
        if (g_out && g_stride < 7 + b->max_tors) throw Error(UD_ERR_ARG, "g_stride smaller than 7 + max torsions");
        if (dw_out && dw_stride < b->maps->sf.n_terms) throw Error(UD_ERR_ARG, "dw_stride smaller than term count");
        if (n_poses == 0) return;
        cudaStream_t s = (cudaStream_t)stream;
        if (dw_out) ensure_terms(b->maps, s);
        DeviceTermsView tv = b->maps->terms_built ? terms_view(b->maps) : DeviceTermsView{nullptr, nullptr, 0, 0, 0};
        cuda_check(launch_adjoint(b->view(), maps_view(b->maps), tables_view(b->maps), tv, (int)b->desc.size(),
                                  pose_ligand, poses, pose_stride, n_poses, v_intra, v_inter,
                                  (flags & UD_ADJOINT_EXACT) ? 1 : 0, e_out, g_out, g_stride, dw_out, dw_stride, s),
                   "adjoint kernel");
    });
}

extern "C" int ud_score_adjoint(ud_batch b, const int* pose_ligand, const float* poses, int n_poses,
                                int pose_stride, float v_intra, float v_inter, int flags, float* e_out, float* g_out,
                                int g_stride, float* dw_out, int dw_stride, void* stream) {
    return guarded([&] {
        check_poses(b, pose_ligand, n_poses, pose_stride);
        if (!poses || !e_out) throw Error(UD_ERR_ARG, "null buffer");
        if (g_out && g_stride < 7 + b->max_tors) throw Error(UD_ERR_ARG, "g_stride smaller than 7 + max torsions");
        const int nt = b->maps->sf.n_terms;
        if (dw_out && dw_stride < nt) throw Error(UD_ERR_ARG, "dw_stride smaller than term count");
        for (int i = 0; i < n_poses; ++i)
            if (pose_ligand[i] < 0 || pose_ligand[i] >= (int)b->desc.size())
                throw Error(UD_ERR_ARG, "pose_ligand out of range");
        if (n_poses == 0) return;
        cudaStream_t s = (cudaStream_t)stream;
        if (dw_out) ensure_terms(b->maps, s);
        b->d_pose_lig.upload(pose_ligand, n_poses, s);
        b->d_pose.upload(poses, (size_t)n_poses * pose_stride, s);
        b->d_e.alloc(n_poses);
        if (g_out) {  // entries past a pose's 7 + T gradient floats come back as 0
            b->d_g.alloc((size_t)n_poses * g_stride);
            cuda_check(cudaMemsetAsync(b->d_g.p, 0, (size_t)n_poses * g_stride * sizeof(float), s), "memset");
        }
        if (dw_out) b->d_dw.alloc((size_t)n_poses * dw_stride);
        DeviceTermsView tv = b->maps->terms_built ? terms_view(b->maps) : DeviceTermsView{nullptr, nullptr, 0, 0, 0};
        cuda_check(launch_adjoint(b->view(), maps_view(b->maps), tables_view(b->maps), tv, (int)b->desc.size(),
                                  b->d_pose_lig.p, b->d_pose.p, pose_stride, n_poses, v_intra, v_inter,
                                  (flags & UD_ADJOINT_EXACT) ? 1 : 0, b->d_e.p, g_out ? b->d_g.p : nullptr, g_stride,
                                  dw_out ? b->d_dw.p : nullptr, dw_stride, s),
                   "adjoint kernel");
        cuda_check(cudaMemcpyAsync(e_out, b->d_e.p, n_poses * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
        if (g_out)
            cuda_check(cudaMemcpyAsync(g_out, b->d_g.p, (size_t)n_poses * g_stride * sizeof(float),
                                       cudaMemcpyDeviceToHost, s),
                       "D2H");
        if (dw_out)
            cuda_check(cudaMemcpyAsync(dw_out, b->d_dw.p, (size_t)n_poses * dw_stride * sizeof(float),
                                       cudaMemcpyDeviceToHost, s),
                       "D2H");
        cuda_check(cudaStreamSynchronize(s), "adjoint sync");
    });
}

// ---------------------------------------------------------------- search

// MC steps per chain (vina.h:187-204): 70*3*(50 + max(atoms + 10*dof))/2,
// capped by max_step.
static int global_steps_for(const std::vector<const Ligand*>& ligs, int max_step) {
    size_t heuristic = 0;
    for (auto* L : ligs) heuristic = std::max(heuristic, L->atoms.size() + 10 * (size_t)(6 + L->n_torsions()));
    unsigned gs = (unsigned)(70 * 3 * (50 + heuristic) / 2);
    if (max_step > 0 && gs > (unsigned)max_step) gs = (unsigned)max_step;
    return (int)gs;
}

static float rmsd_ub(const std::vector<float>& a, const std::vector<float>& b) {
    double acc = 0;
    size_t n = a.size() / 3;
    float accf = 0;
    for (size_t i = 0; i < n; ++i) {
        float dx = a[3 * i] - b[3 * i], dy = a[3 * i + 1] - b[3 * i + 1], dz = a[3 * i + 2] - b[3 * i + 2];
        accf += dx * dx + dy * dy + dz * dz;
    }
    (void)acc;
    return n > 0 ? std::sqrt(accf / n) : 0.0f;
}

// add_to_output_container (unidock/src/lib/coords.cpp:44-68)
static std::vector<float> heavy_coords(const Ligand& L, const std::vector<float>& all) {
    std::vector<float> h;
    for (size_t i = 0; i < L.atoms.size(); ++i)
        if (L.atoms[i].el != EL_H)
            for (int k = 0; k < 3; ++k) h.push_back(all[3 * i + k]);
    return h;
}

static float rmsd_lb_asym(const Ligand& L, const std::vector<float>& x, const std::vector<float>& y) {
    float sum = 0;
    unsigned cnt = 0;
    for (size_t i = 0; i < L.atoms.size(); ++i) {
        if (L.atoms[i].el == EL_H) continue;
        float r2 = std::numeric_limits<float>::max();
        for (size_t j = 0; j < L.atoms.size(); ++j) {
            const Atom& b = L.atoms[j];
            if (L.atoms[i].el == b.el && !(b.ad == AD_H || b.ad == AD_HD)) {
                float dx = x[3 * i] - y[3 * j], dy = x[3 * i + 1] - y[3 * j + 1], dz = x[3 * i + 2] - y[3 * j + 2];
                r2 = std::min(r2, dx * dx + dy * dy + dz * dz);
            }
        }
        sum += r2;
        ++cnt;
    }
    return cnt ? std::sqrt(sum / cnt) : 0.0f;
}

// Runs body(i) for i in [0, n) on the host's hardware threads (dynamic chunks of one).
template <class F> static void parallel_for(int n, F&& body) {
    int nt = (int)std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 64u);
    nt = std::min(nt, std::max(1, n / 4));
    if (nt <= 1) {
        for (int i = 0; i < n; ++i) body(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> ts;
    for (int t = 0; t < nt; ++t)
        ts.emplace_back([&] {
            for (int i = next.fetch_add(1); i < n; i = next.fetch_add(1)) body(i);
        });
    for (auto& t : ts) t.join();
}

// Receptor atoms of the maps in box cells (DeviceReceptorView): the scoring
// without maps that the reference keeps unless --no_refine (non_cache,
// non_cache.cpp:23-30; its szv_grid lists, per cell, the receptor atoms within
// the cutoff of the cell).  2 A cells over the box; atoms listed in receptor
// order.
static bool has_receptor(const ud_maps_s* m) { return !m->desc.ad4 && !m->loaded && !m->rec_xyzt.empty(); }

static void ensure_receptor(ud_maps_s* m, cudaStream_t s) {
    if (m->rc_built) return;
    if (!has_receptor(m))
        throw Error(UD_ERR_STATE, "receptor-atom scoring needs Vina / Vinardo maps built from a receptor");
    const MapsDesc& d = m->desc;
    const float cell = 2.0f;
    DeviceReceptorView& R = m->rc;
    for (int i = 0; i < 3; ++i) {
        R.begin[i] = d.init[i];
        R.end[i] = d.corner2[i];
        R.n[i] = std::max(1, (int)std::ceil((R.end[i] - R.begin[i]) / cell));
    }
    R.inv_cell = 1.0f / cell;
    // margin over the cutoff: a query point on a cell face must not miss an atom by rounding
    const float cut = std::sqrt(m->cutoff2) + 1e-3f, cut2 = cut * cut;
    const int n_rec = (int)(m->rec_xyzt.size() / 4);
    const float* X = m->rec_xyzt.data();
    auto box_d2 = [&](const float* p, const float* lo, const float* hi) {
        float d2 = 0;
        for (int k = 0; k < 3; ++k) {
            const float t = p[k] < lo[k] ? lo[k] - p[k] : (p[k] > hi[k] ? p[k] - hi[k] : 0.0f);
            d2 += t * t;
        }
        return d2;
    };
    const int nx = R.n[0], ny = R.n[1], nz = R.n[2];
    std::vector<std::vector<int>> lists((size_t)nx * ny * nz);
    parallel_for(ny * nz, [&](int row) {
        const int iy = row % ny, iz = row / ny;
        const float lo[3] = {R.begin[0], R.begin[1] + iy * cell, R.begin[2] + iz * cell};
        const float hi[3] = {R.begin[0] + nx * cell, lo[1] + cell, lo[2] + cell};
        std::vector<int> cand;
        for (int a = 0; a < n_rec; ++a)
            if (box_d2(X + 4 * a, lo, hi) < cut2) cand.push_back(a);
        for (int ix = 0; ix < nx; ++ix) {
            const float clo[3] = {R.begin[0] + ix * cell, lo[1], lo[2]};
            const float chi[3] = {clo[0] + cell, hi[1], hi[2]};
            auto& L = lists[((size_t)iz * ny + iy) * nx + ix];
            for (int a : cand)
                if (box_d2(X + 4 * a, clo, chi) < cut2) L.push_back(a);
        }
    });
    std::vector<int> start(lists.size() + 1, 0);
    for (size_t c = 0; c < lists.size(); ++c) start[c + 1] = start[c] + (int)lists[c].size();
    std::vector<float> atoms(4 * (size_t)start.back());
    for (size_t c = 0; c < lists.size(); ++c)
        for (size_t k = 0; k < lists[c].size(); ++k)
            std::memcpy(&atoms[4 * ((size_t)start[c] + k)], X + 4 * (size_t)lists[c][k], 4 * sizeof(float));
    m->rc_atoms.upload(atoms.data(), atoms.size(), s);
    m->rc_start.upload(start.data(), start.size(), s);
    cuda_check(cudaStreamSynchronize(s), "receptor cells");
    R.atoms = m->rc_atoms.p;
    R.start = m->rc_start.p;
    m->rc_built = true;
}

// Whether a search with these parameters refines its modes against the
// receptor atoms (Vina / Vinardo with a receptor, refine_step > 0: the
// reference's default, vina.h:251-272).
static bool refines(const ud_batch b, const ud_search_params& P) {
    return P.refine_step > 0 && has_receptor(b->maps);
}

// The device part after the search kernel: clustering of every ligand's
// chains into modes, their refinement against the receptor atoms and final
// scoring energies when `b->refined`, and the copies of the modes into
// page-locked memory.  Enqueued on `s` (also inside a graph capture).
static cudaError_t enqueue_modes(ud_batch b, cudaStream_t s) {
    const int n_lig = (int)b->ligs.size(), cap = b->mode_cap;
    const size_t n_slot = (size_t)n_lig * cap;
    cudaError_t e = launch_cluster(b->view(), b->d_poses.p, b->pose_stride, b->d_results.p, n_lig, b->exhaustiveness,
                                   cap, b->params.min_rmsd, b->d_cluster_scratch.p, b->d_n_modes.p,
                                   b->d_mode_chain.p, b->d_mode_lig.p, b->d_mode_pose.p, s);
    if (e == cudaSuccess && b->refined)
        e = launch_receptor(kRecRefine, b->view(), tables_view(b->maps), receptor_view(b), b->d_mode_lig.p,
                            b->d_mode_pose.p, b->pose_stride, (int)n_slot, b->params.refine_step, 0.0f, 1000.0f,
                            nullptr, nullptr, 0, b->d_mode_e.p, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->hp_n_modes.p, b->d_n_modes.p, n_lig * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->hp_mode_chain.p, b->d_mode_chain.p, n_slot * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->hp_mode_pose.p, b->d_mode_pose.p, n_slot * b->pose_stride * sizeof(float),
                            cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && b->refined)
        e = cudaMemcpyAsync(b->hp_mode_e.p, b->d_mode_e.p, n_slot * 4 * sizeof(float), cudaMemcpyDeviceToHost, s);
    return e;
}

// Buffers of enqueue_modes for the batch's current parameters.
static void alloc_modes(ud_batch b, cudaStream_t s) {
    const int n_lig = (int)b->ligs.size();
    b->mode_cap = std::max(1, b->params.num_modes);
    b->refined = refines(b, b->params);
    if (b->refined) {
        ensure_receptor(b->maps, s);
        upload_lig_bias(b, s);
    }
    const size_t n_slot = (size_t)n_lig * b->mode_cap;
    b->d_cluster_scratch.alloc(n_slot * 3 * std::max(1, b->max_atoms));
    b->d_n_modes.alloc(n_lig);
    b->d_mode_chain.alloc(n_slot);
    b->d_mode_lig.alloc(n_slot);
    b->d_mode_pose.alloc(n_slot * b->pose_stride);
    b->d_mode_e.alloc(n_slot * 4);
    b->hp_n_modes.alloc(n_lig);
    b->hp_mode_chain.alloc(n_slot);
    b->hp_mode_pose.alloc(n_slot * b->pose_stride);
    b->hp_mode_e.alloc(n_slot * 4);
}

// Final scores of one ligand's modes (vina.h:232-343) from the device
// clustering (and refinement), in mode slots of `cap` per ligand: without
// refinement the modes keep their search order and their grid /
// intramolecular energies at the authentic cap; with it they are ordered by
// refined energy (max when outside the box), and the inter energies come from
// the receptor atoms.  Vina / Vinardo: the final score is conf_independent(
// inter + intra - intra of the first mode) and the unbound energy that first
// mode's intramolecular energy; AD4: inter plus the torsional term, unbound
// -intra (score_gpu, vina.cpp:1245-1322).
static LigandPost post_process_ligand(const Scoring& sf, const Ligand& L, int E, int cap, int pose_stride,
                                      bool refined, int n_modes, const int* mode_chain, const float* mode_pose,
                                      const float* mode_e, const ChainResult* results) {
        LigandPost out;
        std::vector<PoseResult> v;
        for (int k = 0; k < n_modes; ++k) {
            const int ch = mode_chain[k];
            const ChainResult& cr = results[ch];
            PoseResult r;
            const float* p = mode_pose + (size_t)k * pose_stride;
            r.pose.assign(p, p + 7 + L.n_torsions());
            if (refined) {
                const float* me = mode_e + 4 * (size_t)k;
                r.e = me[3] > 0.5f ? me[0] : std::numeric_limits<float>::max();
                r.inter = me[1];
                r.intra = me[2];
            } else {
                r.e = cr.e;
                r.inter = cr.e_grid;
                r.intra = cr.e_intra;
            }
            v.push_back(r);
        }
        if (v.empty()) return out;
        if (refined)
            std::stable_sort(v.begin(), v.end(), [](const PoseResult& x, const PoseResult& y) { return x.e < y.e; });
        auto ci = L.conf_indep_inputs();
        const bool ad4 = sf.choice == SF_AD42;
        const float intramolecular = v[0].intra;
        for (size_t i = 0; i < v.size(); ++i) {
            const float inter = v[i].inter, intra = v[i].intra;
            if (ad4) {  // score_gpu's AD4 branch (vina.cpp:1290-1322): inter + torsional term, unbound -intra
                const float tors = sf.conf_independent(0.0f, ci[0], (float)L.torsdof);
                v[i].e = inter + tors;
                v[i].conf_indep = tors;
                v[i].unbound = -intra;
            } else {
                const float total = sf.conf_independent(inter + intra - intramolecular, ci[0], (float)L.torsdof);
                v[i].e = total;
                v[i].conf_indep = total - (inter + intra - intramolecular);
                v[i].unbound = intramolecular;
            }
            v[i].inter = inter;
            v[i].intra = intra;
            v[i].total = inter + intra;
        }
        std::stable_sort(v.begin(), v.end(), [](const PoseResult& x, const PoseResult& y) { return x.e < y.e; });
        std::vector<float> best(3 * L.atoms.size()), cur(3 * L.atoms.size());
        ligand_coords(L, v[0].pose.data(), best.data());
        for (auto& r : v) {
            ligand_coords(L, r.pose.data(), cur.data());
            r.lb = std::max(rmsd_lb_asym(L, cur, best), rmsd_lb_asym(L, best, cur));
            r.ub = rmsd_ub(heavy_coords(L, cur), heavy_coords(L, best));
        }
        out.modes = std::move(v);
        return out;
}

// Final scores of every ligand of the batch (post_process_ligand), on the
// host's threads.
static void post_process(ud_batch b) {
    const int n_lig = (int)b->ligs.size();
    const int E = b->exhaustiveness, cap = b->mode_cap;
    b->post.assign(n_lig, LigandPost{});
    parallel_for(n_lig, [&](int l) {
        const size_t o = (size_t)l * cap;
        b->post[l] = post_process_ligand(b->maps->sf, *b->ligs[l], E, cap, b->pose_stride, b->refined,
                                         b->hp_n_modes.p[l], b->hp_mode_chain.p + o,
                                         b->hp_mode_pose.p + o * b->pose_stride, b->hp_mode_e.p + 4 * o,
                                         b->h_results.data() + (size_t)l * E);
    });
}

// Capture (or reuse) the per-batch sequence of the persistent search as a
// CUDA graph: queue reset, search kernel, results into page-locked memory,
// clustering (and refinement) of the modes and their copies.
// Captured on the batch's own stream (capture is not allowed on the legacy
// default stream); the instantiated graph is then launched on any stream.
// Reused while the launch parameters and buffers are unchanged.
static void search_graph(ud_batch b, const SearchParams& sp, int n_chain, int blocks) {
    b->hp_poses.alloc((size_t)n_chain * b->pose_stride);
    b->hp_results.alloc((size_t)n_chain);
    std::ostringstream k;
    k << n_chain << ' ' << blocks << ' ' << sp.global_steps << ' ' << sp.exhaustiveness << ' ' << sp.seed << ' '
      << sp.chains_per_block << ' ' << sp.lanes_per_chain << ' ' << sp.bfgs_cap << ' ' << (const void*)b->d_poses.p << ' '
      << (const void*)b->d_results.p << ' ' << (const void*)b->d_queue.p << ' ' << (const void*)b->d_order.p << ' '
      << (const void*)b->hp_poses.p << ' ' << (const void*)b->hp_results.p << ' ' << (const void*)b->maps->maps.p << ' ' << (const void*)b->maps->xpairs.p
      << ' ' << (const void*)b->maps->smooth.p << ' ' << b->mode_cap << ' ' << b->refined << ' '
      << b->params.refine_step << ' ' << b->params.min_rmsd << ' ' << (const void*)b->d_mode_pose.p << ' '
      << (const void*)b->d_mode_e.p << ' ' << (const void*)b->d_cluster_scratch.p << ' '
      << (const void*)b->hp_mode_pose.p << ' ' << (const void*)b->hp_mode_e.p << ' ' << (const void*)b->hp_n_modes.p
      << ' ' << (const void*)b->hp_mode_chain.p << ' ' << (const void*)b->maps->rc.atoms << ' '
      << (const void*)b->maps->rc.start << ' ' << (const void*)b->maps->rc.bias << ' ' << b->maps->rc.n_bias << ' '
      << (const void*)receptor_view(b).lig_bias << ' ' << (const void*)receptor_view(b).lig_bias_span << ' '
      << (const void*)b->maps->fast.p << ' '
      << (const void*)b->d_n_modes.p << ' ' << (const void*)b->d_mode_chain.p << ' ' << (const void*)b->d_mode_lig.p;
    // the topology (reallocated when a reused handle gets a larger batch) and
    // the per-warp shared-memory layout it sizes
    const DeviceBatchView v = b->view();
    k << ' ' << (const void*)v.ligs << ' ' << (const void*)v.atoms << ' ' << (const void*)v.nodes << ' '
      << (const void*)v.pairs << ' ' << (const void*)v.grid_list << ' '
      << (const void*)v.charges << ' '
      << (const void*)v.pair_coef << ' ' << v.max_atoms << ' ' << v.max_torsions << ' ' << b->ligs.size() << ' '
      << b->pose_stride;
    if (b->graph_exec && b->graph_key == k.str()) return;
    b->drop_graph();
    if (!b->capture_stream)
        cuda_check(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking), "capture stream");
    cudaStream_t cs = b->capture_stream;
    cuda_check(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t e = cudaMemsetAsync(b->d_queue.p, 0, sizeof(unsigned int), cs);
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(b->evk0, cs, cudaEventRecordExternal);
    if (e == cudaSuccess)
        e = launch_search(b->view(), maps_view(b->maps), tables_view(b->maps), sp, b->d_order.p, n_chain, 0,
                          b->d_queue.p, b->d_poses.p, b->pose_stride, b->d_results.p, blocks, cs);
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(b->evk1, cs, cudaEventRecordExternal);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->hp_poses.p, b->d_poses.p, (size_t)n_chain * b->pose_stride * sizeof(float),
                            cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->hp_results.p, b->d_results.p, (size_t)n_chain * sizeof(ChainResult),
                            cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = enqueue_modes(b, cs);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cs, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cuda_check(e != cudaSuccess ? e : e2, "search graph capture");
    }
    b->graph = g;
    cuda_check(cudaGraphInstantiate(&b->graph_exec, g, 0), "graph instantiate");
    b->graph_key = k.str();
}

// Launch the search kernels of the batch asynchronously on `s`, followed by the
// clustering (and refinement) of the modes unless `modes` is false.
// `launch` false: only the set-up (buffers, ligand order, graph capture).
// CTA size (warps) of a persistent search whose caller and autotuner gave
// none: of 4, 2 and 1 warps, the one that keeps the most chains resident per
// SM at the batch's layout, ties to the larger CTA.  A large layout, whose
// per-chain shared memory lets few 4-warp CTAs onto an SM, gets smaller CTAs.
static int default_chains_per_block(const DeviceBatchView& v, int lanes, bool stream) {
    int best = 4, best_resident = 0;
    for (int w : {4, 2, 1}) {
        const int per_sm = stream ? stream_blocks_per_sm(v, w) : search_blocks_per_sm(v, w, lanes);
        if (per_sm * w > best_resident) {
            best = w;
            best_resident = per_sm * w;
        }
    }
    return best;
}

static void search_launch(ud_batch b, const ud_search_params* params, cudaStream_t s, bool launch = true,
                          bool modes = true) {
        if (!b || !params) throw Error(UD_ERR_ARG, "null argument");
        const ud_search_params& P = *params;
        if (P.exhaustiveness < 1) throw Error(UD_ERR_ARG, "exhaustiveness must be >= 1");
        if (P.chains_per_block < 0 || P.chains_per_block > 4)
            throw Error(UD_ERR_ARG, "chains_per_block must be 0 (default / autotuned) or 1..4");
        if (P.lanes_per_chain != 0 && P.lanes_per_chain != 16 && P.lanes_per_chain != 32)
            throw Error(UD_ERR_ARG, "lanes_per_chain must be 0 (default / autotuned), 16 or 32");
        if (P.num_modes < 1) throw Error(UD_ERR_ARG, "num_modes must be >= 1");
        const int n_lig = (int)b->ligs.size();
        if (n_lig == 0) throw Error(UD_ERR_ARG, "empty batch");
        b->params = P;
        b->searched = false;
        b->text_ready[0] = b->text_ready[1] = false;
        const int E = P.exhaustiveness;
        b->exhaustiveness = E;
        b->pose_stride = 7 + b->max_tors;
        const size_t n_chain = (size_t)n_lig * E;
        b->d_poses.alloc(n_chain * b->pose_stride);
        b->d_results.alloc(n_chain);
        b->d_queue.alloc(1);
        if (modes) alloc_modes(b, s);
        SearchParams sp{};
        sp.global_steps = global_steps_for(b->ligs, P.max_step);
        sp.exhaustiveness = E;
        sp.seed = P.seed;
        sp.hunt_cap = 10.0f;
        sp.authentic_v = 1000.0f;
        sp.temperature = 1.2f;
        sp.mutation_amplitude = 2.0f;
        // the plain form keeps one chain per warp (the fixed tiling it stands for)
        sp.lanes_per_chain = P.form != 1 ? 32
                             : P.lanes_per_chain > 0 ? P.lanes_per_chain : (b->tuned ? b->tuned_lanes_per_chain : 32);
        sp.chains_per_block = P.chains_per_block > 0 ? P.chains_per_block
                              : b->tuned                 ? b->tuned_chains_per_block
                              : P.form == 1              ? default_chains_per_block(b->view(), sp.lanes_per_chain, false)
                                                         : 4;
        const int chains_per_cta = sp.chains_per_block * (32 / sp.lanes_per_chain);
        sp.persistent = P.form == 1 ? 1 : 0;
        sp.bfgs_cap = P.bfgs_cap >= 0 ? P.bfgs_cap : (b->tuned ? b->tuned_bfgs_cap : 0);
        int dev = 0, n_sm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        if (!b->ev0) {
            cuda_check(cudaEventCreate(&b->ev0), "event");
            cuda_check(cudaEventCreate(&b->ev1), "event");
            cuda_check(cudaEventCreate(&b->evk0), "event");
            cuda_check(cudaEventCreate(&b->evk1), "event");
        }
        b->graph_results = false;
        if (sp.persistent && P.use_graph && modes) {
            int per_sm = search_blocks_per_sm(b->view(), sp.chains_per_block, sp.lanes_per_chain);
            int blocks = std::max(1, std::min(per_sm * n_sm, (int)((n_chain + chains_per_cta - 1) / chains_per_cta)));
            search_graph(b, sp, (int)n_chain, blocks);
            if (!launch) return;
            cudaEventRecord(b->ev0, s);
            cuda_check(cudaGraphLaunch(b->graph_exec, s), "graph launch");
            cudaEventRecord(b->ev1, s);
            b->graph_results = true;
            b->launched = true;
            return;
        }
        if (!launch) return;
        cudaEventRecord(b->ev0, s);
        if (sp.persistent) {
            cuda_check(cudaMemsetAsync(b->d_queue.p, 0, sizeof(unsigned int), s), "queue reset");
            int per_sm = search_blocks_per_sm(b->view(), sp.chains_per_block, sp.lanes_per_chain);
            int blocks = per_sm * n_sm;
            int needed = (int)((n_chain + chains_per_cta - 1) / chains_per_cta);
            blocks = std::max(1, std::min(blocks, needed));
            cuda_check(launch_search(b->view(), maps_view(b->maps), tables_view(b->maps), sp, b->d_order.p,
                                     (int)n_chain, 0, b->d_queue.p, b->d_poses.p, b->pose_stride, b->d_results.p,
                                     blocks, s),
                       "search kernel");
        } else {
            for (int k = 0; k < n_lig; ++k) {
                cuda_check(launch_search(b->view(), maps_view(b->maps), tables_view(b->maps), sp, b->d_order.p, E,
                                         k * E, b->d_queue.p, b->d_poses.p, b->pose_stride, b->d_results.p, 0, s),
                           "search kernel");
            }
        }
        cudaEventRecord(b->ev1, s);
        if (modes) cuda_check(enqueue_modes(b, s), "modes");
        b->launched = true;
}

// Copy the results of the launched search to the host and finish the modes.
static void search_collect(ud_batch b, cudaStream_t s) {
        if (!b || !b->launched) throw Error(UD_ERR_STATE, "no search launched");
        const size_t n_chain = (size_t)b->ligs.size() * b->exhaustiveness;
        b->h_poses.resize(n_chain * b->pose_stride);
        b->h_results.resize(n_chain);
        if (b->graph_results) {  // the graph copied them into page-locked memory
            cuda_check(cudaStreamSynchronize(s), "search sync");
            std::memcpy(b->h_poses.data(), b->hp_poses.p, b->h_poses.size() * sizeof(float));
            std::memcpy(b->h_results.data(), b->hp_results.p, n_chain * sizeof(ChainResult));
        } else {
            cuda_check(cudaMemcpyAsync(b->h_poses.data(), b->d_poses.p, b->h_poses.size() * sizeof(float),
                                       cudaMemcpyDeviceToHost, s),
                       "D2H poses");
            cuda_check(cudaMemcpyAsync(b->h_results.data(), b->d_results.p, n_chain * sizeof(ChainResult),
                                       cudaMemcpyDeviceToHost, s),
                       "D2H results");
            cuda_check(cudaStreamSynchronize(s), "search sync");
        }
        // the search kernel's own device time: between the graph's event
        // nodes around it, else (no graph) between the events of the launch
        b->kernel_ms = 0;
        if (!b->graph_results || cudaEventElapsedTime(&b->kernel_ms, b->evk0, b->evk1) != cudaSuccess) {
            cudaGetLastError();
            cudaEventElapsedTime(&b->kernel_ms, b->ev0, b->ev1);
        }
        b->evals = 0;
        for (auto& r : b->h_results) b->evals += r.evals;
        post_process(b);
        b->launched = false;
        b->searched = true;
}

// ---------------------------------------------------------------- receptor atoms

static void check_receptor_poses(ud_batch b, const int* pose_ligand, const float* poses, int n_poses,
                                 int pose_stride) {
    check_poses(b, pose_ligand, n_poses, pose_stride);
    if (!poses) throw Error(UD_ERR_ARG, "null buffer");
    for (int i = 0; i < n_poses; ++i)
        if (pose_ligand[i] < 0 || pose_ligand[i] >= (int)b->desc.size())
            throw Error(UD_ERR_ARG, "pose_ligand out of range");
}

// Receptor-atom kernel of `mode` over host poses; out4 (4 floats per pose) read back.
static void receptor_poses(ud_batch b, int mode, const int* pose_ligand, float* poses, int n_poses, int pose_stride,
                           int refine_step, std::vector<float>& out4, cudaStream_t s) {
    ensure_receptor(b->maps, s);
    upload_lig_bias(b, s);
    out4.assign(4 * (size_t)n_poses, 0.0f);
    if (n_poses == 0) return;
    b->d_pose_lig.upload(pose_ligand, n_poses, s);
    b->d_pose.upload(poses, (size_t)n_poses * pose_stride, s);
    b->d_score.alloc(4 * (size_t)n_poses);
    cuda_check(launch_receptor(mode, b->view(), tables_view(b->maps), receptor_view(b), b->d_pose_lig.p, b->d_pose.p,
                               pose_stride, n_poses, refine_step, 0.0f, 1000.0f, nullptr, nullptr, 0, b->d_score.p, s),
               "receptor kernel");
    if (mode == kRecRefine)
        cuda_check(cudaMemcpyAsync(poses, b->d_pose.p, (size_t)n_poses * pose_stride * sizeof(float),
                                   cudaMemcpyDeviceToHost, s),
                   "D2H");
    cuda_check(cudaMemcpyAsync(out4.data(), b->d_score.p, 4 * (size_t)n_poses * sizeof(float),
                               cudaMemcpyDeviceToHost, s),
               "D2H");
    cuda_check(cudaStreamSynchronize(s), "receptor sync");
}

extern "C" int ud_score_grad_receptor(ud_batch b, const int* pose_ligand, const float* poses, int n_poses,
                                      int pose_stride, float slope, float v, float* e_out, float* g_out, int g_stride,
                                      void* stream) {
    return guarded([&] {
        check_receptor_poses(b, pose_ligand, poses, n_poses, pose_stride);
        if (!e_out || !g_out || g_stride < 6 + b->max_tors) throw Error(UD_ERR_ARG, "invalid buffers");
        cudaStream_t s = (cudaStream_t)stream;
        ensure_receptor(b->maps, s);
        upload_lig_bias(b, s);
        if (n_poses == 0) return;
        b->d_pose_lig.upload(pose_ligand, n_poses, s);
        b->d_pose.upload(poses, (size_t)n_poses * pose_stride, s);
        b->d_e.alloc(n_poses);
        b->d_g.alloc((size_t)n_poses * g_stride);
        cuda_check(cudaMemsetAsync(b->d_g.p, 0, (size_t)n_poses * g_stride * sizeof(float), s), "memset");
        cuda_check(launch_receptor(kRecEnergyGrad, b->view(), tables_view(b->maps), receptor_view(b), b->d_pose_lig.p,
                                   b->d_pose.p, pose_stride, n_poses, 0, slope, v, b->d_e.p, b->d_g.p, g_stride,
                                   nullptr, s),
                   "receptor kernel");
        cuda_check(cudaMemcpyAsync(e_out, b->d_e.p, n_poses * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaMemcpyAsync(g_out, b->d_g.p, (size_t)n_poses * g_stride * sizeof(float),
                                   cudaMemcpyDeviceToHost, s),
                   "D2H");
        cuda_check(cudaStreamSynchronize(s), "receptor sync");
    });
}

extern "C" int ud_refine(ud_batch b, const int* pose_ligand, float* poses, int n_poses, int pose_stride,
                         int refine_step, float* out4, void* stream) {
    return guarded([&] {
        check_receptor_poses(b, pose_ligand, poses, n_poses, pose_stride);
        if (!out4 || refine_step < 0) throw Error(UD_ERR_ARG, "invalid refinement arguments");
        std::vector<float> o;
        receptor_poses(b, kRecRefine, pose_ligand, poses, n_poses, pose_stride, refine_step, o, (cudaStream_t)stream);
        std::copy(o.begin(), o.end(), out4);
    });
}

extern "C" int ud_score_terms_receptor(ud_batch b, const int* pose_ligand, const float* poses, int n_poses,
                                       int pose_stride, float* out, void* stream) {
    return guarded([&] {
        check_receptor_poses(b, pose_ligand, poses, n_poses, pose_stride);
        if (!out) throw Error(UD_ERR_ARG, "null buffer");
        std::vector<float> p(poses, poses + (size_t)n_poses * pose_stride), o;
        receptor_poses(b, kRecScore, pose_ligand, p.data(), n_poses, pose_stride, 0, o, (cudaStream_t)stream);
        const Scoring& sf = b->maps->sf;
        for (int i = 0; i < n_poses; ++i) {
            const Ligand& L = *b->ligs[pose_ligand[i]];
            const float inter = o[4 * i + 1], intra = o[4 * i + 2];
            const float total = sf.conf_independent(inter + intra - intra, L.conf_indep_inputs()[0], (float)L.torsdof);
            float* r = out + 8 * (size_t)i;
            r[0] = total;
            r[1] = inter;
            r[2] = 0.0f;
            r[3] = 0.0f;
            r[4] = 0.0f;
            r[5] = intra;
            r[6] = total - inter;
            r[7] = intra;
        }
    });
}

// ---------------------------------------------------------------- autotuner

// Per-ligand best chain energy and device time of one search of `tb`.
static float trial_search(ud_batch tb, const ud_search_params& tp, cudaStream_t s, std::vector<float>& best) {
    search_launch(tb, &tp, s, true, false);
    const size_t n_lig = tb->ligs.size(), E = (size_t)tp.exhaustiveness;
    std::vector<ChainResult> r(n_lig * E);
    cuda_check(cudaMemcpyAsync(r.data(), tb->d_results.p, r.size() * sizeof(ChainResult), cudaMemcpyDeviceToHost, s),
               "D2H results");
    cuda_check(cudaStreamSynchronize(s), "trial sync");
    tb->launched = false;
    float ms = 0;
    cudaEventElapsedTime(&ms, tb->ev0, tb->ev1);
    best.assign(n_lig, std::numeric_limits<float>::max());
    for (size_t i = 0; i < r.size(); ++i) best[i / E] = std::min(best[i / E], r[i].e);
    return ms;
}

extern "C" int ud_autotune(ud_batch b, const ud_search_params* params, ud_tune_result* out, void* stream) {
    return guarded([&] {
        if (!b || !params || !out) throw Error(UD_ERR_ARG, "null argument");
        if (params->exhaustiveness < 1) throw Error(UD_ERR_ARG, "exhaustiveness must be >= 1");
        cudaStream_t s = (cudaStream_t)stream;
        const int n_lig = (int)b->ligs.size();
        if (n_lig == 0) throw Error(UD_ERR_ARG, "empty batch");
        const int E = params->exhaustiveness;
        // sample: ligands spread evenly over the cost order, enough chains to
        // fill every SM's resident warps about twice
        std::vector<int> order(n_lig);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            long long cx = (long long)b->desc[x].local_steps * (b->desc[x].n_atoms + b->desc[x].n_pairs);
            long long cy = (long long)b->desc[y].local_steps * (b->desc[y].n_atoms + b->desc[y].n_pairs);
            return cx > cy;
        });
        int dev = 0, n_sm = 148;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        cuda_check(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev), "device attribute");
        // chains resident at once with two chains per warp (the larger count)
        const long long resident = (long long)search_blocks_per_sm(b->view(), 4, 16) * n_sm * 8;
        const int S = (int)std::max<long long>(1, std::min<long long>({(2 * resident + E - 1) / E, n_lig, 512}));
        std::vector<const Ligand*> sample;
        for (int i = 0; i < S; ++i) sample.push_back(b->ligs[order[(size_t)i * n_lig / S]]);
        auto tb = build_batch(b->maps, sample, s);
        ud_search_params tp = *params;
        tp.form = 1;
        tp.use_graph = 0;
        // tuning budget: the caller's MC step cap, or at most 40 steps per chain
        if (tp.max_step <= 0 || tp.max_step > 40) tp.max_step = 40;
        // BFGS iteration caps are not tuned: every cap tried (16, 10, 6) moved the
        // median best energy of the fast screen (exhaustiveness 128, max_step 20)
        // away from the reference's uncapped search by more than 0.1 kcal/mol
        // beyond sampling noise; searches stay uncapped unless bfgs_cap asks.
        const int cpbs[] = {4, 2, 1};
        const int lanes[] = {32, 16};
        std::vector<float> base, cur;
        tp.chains_per_block = 4;
        tp.lanes_per_chain = 32;
        tp.bfgs_cap = 0;
        trial_search(tb.get(), tp, s, cur);                 // warm-up (module load, caches)
        float base_ms = trial_search(tb.get(), tp, s, base);
        int best_cpb = 4, best_lanes = 32, best_cap = 0, tried = 1;
        float best_ms = base_ms, best_shift = 0.0f;
        auto trial = [&](int cpb, int ln, int cap) {
            tp.chains_per_block = cpb;
            tp.lanes_per_chain = ln;
            tp.bfgs_cap = cap;
            const float ms = trial_search(tb.get(), tp, s, cur);
            ++tried;
            double shift = 0;
            for (int i = 0; i < S; ++i) shift += (double)cur[i] - (double)base[i];
            shift /= S;
            // accept only configurations whose search quality holds and that
            // beat the best so far by more than the sample's timing noise
            if (shift <= 0.1 && ms < 0.97f * best_ms) {
                best_ms = ms;
                best_cpb = cpb;
                best_lanes = ln;
                best_cap = cap;
                best_shift = (float)shift;
            }
        };
        // the launch shape: warps per CTA x lanes per chain
        for (int ln : lanes)
            for (int cpb : cpbs)
                if (!(cpb == 4 && ln == 32)) trial(cpb, ln, 0);
        b->tuned = true;
        b->tuned_chains_per_block = best_cpb;
        b->tuned_lanes_per_chain = best_lanes;
        b->tuned_bfgs_cap = best_cap;
        out->chains_per_block = best_cpb;
        out->lanes_per_chain = best_lanes;
        out->bfgs_cap = best_cap;
        out->n_sample = S;
        out->n_tried = tried;
        out->ligands_per_s = best_ms > 0 ? 1e3f * S / best_ms : 0.0f;
        out->base_ligands_per_s = base_ms > 0 ? 1e3f * S / base_ms : 0.0f;
        out->energy_shift = best_shift;
    });
}

extern "C" int ud_search(ud_batch b, const ud_search_params* params, void* stream) {
    return guarded([&] {
        search_launch(b, params, (cudaStream_t)stream);
        search_collect(b, (cudaStream_t)stream);
    });
}

extern "C" int ud_search_prepare(ud_batch b, const ud_search_params* params, void* stream) {
    return guarded([&] {
        search_launch(b, params, (cudaStream_t)stream, false);
        cuda_check(cudaStreamSynchronize((cudaStream_t)stream), "prepare sync");
    });
}

extern "C" int ud_search_launch(ud_batch b, const ud_search_params* params, void* stream) {
    return guarded([&] { search_launch(b, params, (cudaStream_t)stream); });
}

extern "C" int ud_search_collect(ud_batch b, void* stream) {
    return guarded([&] { search_collect(b, (cudaStream_t)stream); });
}

extern "C" int ud_search_chains(ud_batch b, float* poses, int pose_stride, float* e, int* evals) {
    return guarded([&] {
        if (!b || !b->searched) throw Error(UD_ERR_STATE, "no search results");
        const size_t n = b->h_results.size();
        for (size_t i = 0; i < n; ++i) {
            if (e) e[i] = b->h_results[i].e;
            if (evals) evals[i] = b->h_results[i].evals;
            if (poses) {
                if (pose_stride < b->pose_stride) throw Error(UD_ERR_ARG, "pose_stride too small");
                std::copy(&b->h_poses[i * b->pose_stride], &b->h_poses[i * b->pose_stride] + b->pose_stride,
                          poses + i * pose_stride);
            }
        }
    });
}

extern "C" int ud_result_count(ud_batch b, int lig, int* n_modes) {
    return guarded([&] {
        if (!b || !b->searched) throw Error(UD_ERR_STATE, "no search results");
        if (lig < 0 || lig >= (int)b->post.size() || !n_modes) throw Error(UD_ERR_ARG, "ligand out of range");
        *n_modes = (int)b->post[lig].modes.size();
    });
}

extern "C" int ud_result_mode(ud_batch b, int lig, int k, float* pose, float energies[8]) {
    return guarded([&] {
        if (!b || !b->searched) throw Error(UD_ERR_STATE, "no search results");
        if (lig < 0 || lig >= (int)b->post.size()) throw Error(UD_ERR_ARG, "ligand out of range");
        const auto& m = b->post[lig].modes;
        if (k < 0 || k >= (int)m.size()) throw Error(UD_ERR_ARG, "mode out of range");
        if (pose) std::copy(m[k].pose.begin(), m[k].pose.end(), pose);
        if (energies) {
            energies[0] = m[k].e;
            energies[1] = m[k].lb;
            energies[2] = m[k].ub;
            energies[3] = m[k].total;
            energies[4] = m[k].inter;
            energies[5] = m[k].intra;
            energies[6] = m[k].conf_indep;
            energies[7] = m[k].unbound;
        }
    });
}

// Output text of one ligand: the kept modes within num_modes and energy_range
// of the best (Vina::get_poses_gpu, vina.cpp:872-923).
static std::string render_modes(const Ligand& L, const LigandPost& post, int num_modes, float energy_range, bool ad4,
                                int format) {
    const auto& modes = post.modes;
    std::vector<PoseResult> sel;
    if (!modes.empty()) {
        const float best = modes[0].e;
        for (auto& m : modes) {
            if ((int)sel.size() >= num_modes) break;
            if (!(m.e < 0.1f * std::numeric_limits<float>::max()) || m.e > best + energy_range) break;
            sel.push_back(m);
        }
    }
    return format == 1 ? write_sdf_models(L, sel, ad4) : write_pdbqt_models(L, sel, ad4);
}

static std::string render_result(const ud_batch_s* b, int lig, int format) {
    return render_modes(*b->ligs[lig], b->post[lig], b->params.num_modes, b->params.energy_range,
                        b->maps->desc.ad4 != 0, format);
}

extern "C" int ud_result_write(ud_batch b, int lig, int format, char* buf, size_t cap, size_t* len) {
    return guarded([&] {
        if (!b || !b->searched) throw Error(UD_ERR_STATE, "no search results");
        if (lig < 0 || lig >= (int)b->post.size()) throw Error(UD_ERR_ARG, "ligand out of range");
        if (format != 0 && format != 1) throw Error(UD_ERR_ARG, "format must be 0 (PDBQT) or 1 (SDF)");
        if (!b->text_ready[format]) {  // every ligand's text at once, on all host threads
            auto& t = b->text[format];
            t.assign(b->post.size(), std::string());
            parallel_for((int)t.size(), [&](int i) { t[i] = render_result(b, i, format); });
            b->text_ready[format] = true;
        }
        const std::string& s = b->text[format][lig];
        if (len) *len = s.size();
        if (buf && cap > 0) {
            size_t n = std::min(cap - 1, s.size());
            std::memcpy(buf, s.data(), n);
            buf[n] = 0;
        }
    });
}

extern "C" int ud_batch_upload_bytes(ud_batch b, size_t* bytes) {
    return guarded([&] {
        if (!b || !bytes) throw Error(UD_ERR_ARG, "null argument");
        *bytes = b->upload_bytes;
    });
}

extern "C" int ud_search_stats(ud_batch b, long long* evals, float* kernel_ms) {
    return guarded([&] {
        if (!b || !b->searched) throw Error(UD_ERR_STATE, "no search results");
        if (evals) *evals = b->evals;
        if (kernel_ms) *kernel_ms = b->kernel_ms;
    });
}

extern "C" int ud_optimize(ud_batch b, const int* pose_ligand, float* poses, int n_poses, int pose_stride,
                           int max_steps, float v, float* e_out, int* evals_out, void* stream) {
    return guarded([&] {
        check_poses(b, pose_ligand, n_poses, pose_stride);
        if (!poses || !e_out) throw Error(UD_ERR_ARG, "null buffer");
        for (int i = 0; i < n_poses; ++i)
            if (pose_ligand[i] < 0 || pose_ligand[i] >= (int)b->desc.size())
                throw Error(UD_ERR_ARG, "pose_ligand out of range");
        if (n_poses == 0) return;
        cudaStream_t s = (cudaStream_t)stream;
        b->d_pose_lig.upload(pose_ligand, n_poses, s);
        b->d_pose.upload(poses, (size_t)n_poses * pose_stride, s);
        b->d_e.alloc(n_poses);
        DevBuf<int> d_ev;
        d_ev.alloc(n_poses);
        cuda_check(launch_optimize(b->view(), maps_view(b->maps), tables_view(b->maps), b->d_pose_lig.p, b->d_pose.p,
                                   pose_stride, n_poses, max_steps, v, b->d_e.p, d_ev.p, s),
                   "optimize kernel");
        cuda_check(cudaMemcpyAsync(poses, b->d_pose.p, (size_t)n_poses * pose_stride * sizeof(float),
                                   cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaMemcpyAsync(e_out, b->d_e.p, n_poses * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
        std::vector<int> ev(n_poses);
        cuda_check(cudaMemcpyAsync(ev.data(), d_ev.p, n_poses * sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaStreamSynchronize(s), "optimize sync");
        if (evals_out) std::copy(ev.begin(), ev.end(), evals_out);
    });
}

extern "C" int ud_device_fp32_peak(float* tflops) {
    return guarded([&] {
        if (!tflops) throw Error(UD_ERR_ARG, "null argument");
        *tflops = measure_fp32_peak_tflops();
        if (!(*tflops > 0)) throw Error(UD_ERR_CUDA, "fp32 probe failed");
    });
}

extern "C" int ud_device_l2_peak(float* gbs) {
    return guarded([&] {
        if (!gbs) throw Error(UD_ERR_ARG, "null argument");
        *gbs = measure_l2_read_gbs();
        if (!(*gbs > 0)) throw Error(UD_ERR_CUDA, "L2 probe failed");
    });
}

// Persistent search with caller-provided device outputs and the library's
// static device scratch instead of device allocations (see the header).  The
// launch shape and BFGS cap resolve as ud_search resolves them for the
// batched form, so both give the same per-chain results.
extern "C" int ud_search_device_noalloc(ud_batch b, const ud_search_params* params, float* d_poses,
                                        int pose_stride, float* d_energies, int* d_evals, void* stream) {
    return guarded([&] {
        if (!b || !params || !d_poses || !d_energies) throw Error(UD_ERR_ARG, "null argument");
        const ud_search_params& P = *params;
        if (P.exhaustiveness < 1) throw Error(UD_ERR_ARG, "exhaustiveness must be >= 1");
        if (P.chains_per_block < 0 || P.chains_per_block > 4)
            throw Error(UD_ERR_ARG, "chains_per_block must be 0 (default / autotuned) or 1..4");
        if (P.lanes_per_chain != 0 && P.lanes_per_chain != 16 && P.lanes_per_chain != 32)
            throw Error(UD_ERR_ARG, "lanes_per_chain must be 0 (default / autotuned), 16 or 32");
        if (pose_stride < 7 + b->max_tors) throw Error(UD_ERR_ARG, "pose_stride smaller than 7 + max torsions");
        const int n_lig = (int)b->ligs.size();
        if (n_lig == 0) throw Error(UD_ERR_ARG, "empty batch");
        const long long n_chain = (long long)n_lig * P.exhaustiveness;
        if (n_chain > kNoAllocMaxChains)
            throw Error(UD_ERR_CAPACITY, "ud_search_device_noalloc: " + std::to_string(n_chain) +
                                             " chains (ligands x exhaustiveness) exceed the maximum of " +
                                             std::to_string(kNoAllocMaxChains));
        SearchParams sp{};
        sp.global_steps = global_steps_for(b->ligs, P.max_step);
        sp.exhaustiveness = P.exhaustiveness;
        sp.seed = P.seed;
        sp.hunt_cap = 10.0f;
        sp.authentic_v = 1000.0f;
        sp.temperature = 1.2f;
        sp.mutation_amplitude = 2.0f;
        sp.lanes_per_chain = P.lanes_per_chain > 0 ? P.lanes_per_chain : (b->tuned ? b->tuned_lanes_per_chain : 32);
        sp.chains_per_block = P.chains_per_block > 0 ? P.chains_per_block
                              : b->tuned ? b->tuned_chains_per_block
                                         : default_chains_per_block(b->view(), sp.lanes_per_chain, false);
        sp.persistent = 1;
        sp.bfgs_cap = P.bfgs_cap >= 0 ? P.bfgs_cap : (b->tuned ? b->tuned_bfgs_cap : 0);
        const int chains_per_cta = sp.chains_per_block * (32 / sp.lanes_per_chain);
        int dev = 0, n_sm = 148;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        cuda_check(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev), "device attribute");
        const int per_sm = search_blocks_per_sm(b->view(), sp.chains_per_block, sp.lanes_per_chain);
        const int needed = (int)((n_chain + chains_per_cta - 1) / chains_per_cta);
        const int blocks = std::max(1, std::min(per_sm * n_sm, needed));
        // the work order (most expensive ligands first) is the batch's own,
        // uploaded to device memory when the batch was filled
        cuda_check(launch_search_noalloc(b->view(), maps_view(b->maps), tables_view(b->maps), sp, b->d_order.p, n_lig,
                                         blocks, d_poses, pose_stride, d_energies, d_evals, (cudaStream_t)stream),
                   "allocation-free search");
    });
}

// ---------------------------------------------------------------- streaming screen
// One persistent search kernel fed slot by slot from the host (StreamView in
// ud_engine.h; no counterpart in the reference, whose CLI parses and docks one
// batch after another, main.cpp:975-1070).  The host packs a slot's ligands
// into page-locked staging memory, copies them into an append-only device
// arena and publishes the slot; the kernel, launched once, takes (ligand,
// chain) items as slots are published and signals each finished slot through
// host-mapped memory; each slot's modes are then clustered and refined on the
// SMs the persistent kernel leaves free, and scored on the host.  Every
// device and page-locked buffer is allocated when the stream is created, so
// nothing synchronises the device while the kernel runs.

namespace {
// A slot's block in every arena array starts on this byte boundary, so that
// no cached line of the read-only data path ever holds a slot that was not
// yet written when the line was cached.
constexpr size_t kSlotAlign = 256;
size_t aligned_elems(size_t n, size_t elem_bytes, size_t unit_elems) {
    (void)elem_bytes;
    return (n + unit_elems - 1) / unit_elems * unit_elems;
}
// elements per alignment unit of each arena array (unit x element size is a
// multiple of kSlotAlign for the array and for the arrays that share its index)
constexpr size_t kAtomUnit = 64;   // AtomRec 16 B (1 KB) and the AD4 charges 4 B (256 B)
constexpr size_t kNodeUnit = 32;   // NodeRec 40 B (1280 B)
constexpr size_t kPairUnit = 64;   // pair words 4 B (256 B) and the AD4 coefficients 8 B (512 B)
constexpr size_t kGridUnit = 64;   // grid-atom words 4 B
constexpr int kStreamReserveSms = 4;  // SMs left to the per-slot clustering and refinement kernels
}  // namespace

struct StreamSlot {
    std::vector<const Ligand*> ligs;
    int max_atoms = 0, max_tors = 0;
    bool collected = false;
    std::vector<LigandPost> post;
    std::vector<ChainResult> results;
    std::vector<float> poses;
};

struct ud_stream_s {
    ud_maps maps = nullptr;
    ud_search_params params{};
    SearchParams sp{};
    int E = 0, M = 0, max_slots = 0, ring = 0, cap = 0, stride = 0, max_atoms = 0, max_tors = 0;
    bool refined = false, ad4 = false;
    size_t atom_cap = 0, node_cap = 0, pair_cap = 0, grid_cap = 0;
    size_t n_atoms = 0, n_nodes = 0, n_pairs = 0, n_grid = 0;  // arena fill, in elements
    DevBuf<LigDesc> d_desc;
    DevBuf<AtomRec> d_atoms;
    DevBuf<NodeRec> d_nodes;
    DevBuf<uint32_t> d_pairs, d_grid;
    DevBuf<float> d_charge, d_coef;
    DevBuf<unsigned int> d_ctl;  // published, closed, work counter
    DevBuf<unsigned int> d_slot_left;
    DevBuf<int> d_slot_nlig, d_order, d_status;
    unsigned int* h_done = nullptr;  // host-mapped, per slot
    PinnedBuf<unsigned int> h_counts;  // [k] = k: sources of the published-count copies; [max_slots + 1] = 1
    PinnedBuf<unsigned char> staging[2];
    cudaEvent_t staged[2] = {nullptr, nullptr};
    DevBuf<float> d_poses;
    DevBuf<ChainResult> d_results;
    // modes of a slot, one set of buffers per ring area
    DevBuf<float> d_scratch, d_mode_pose, d_mode_e;
    DevBuf<int> d_n_modes, d_mode_chain, d_mode_lig;
    PinnedBuf<int> hp_n_modes, hp_mode_chain;
    PinnedBuf<float> hp_mode_pose, hp_mode_e, hp_poses;
    PinnedBuf<ChainResult> hp_results;
    cudaStream_t ks = nullptr, cs = nullptr, ps = nullptr;  // kernel, copies, post-processing
    std::vector<StreamSlot> slots;
    int n_pushed = 0;
    bool closed = false, running = false, finished = false;
    int status = 0;
    long long evals = 0;

    DeviceBatchView view(int slot = -1) const {
        DeviceBatchView v{d_desc.p, d_atoms.p, d_nodes.p, d_pairs.p, d_grid.p, max_atoms, max_tors,
                          d_charge.p, d_coef.p, ad4 ? 1 : 0};
        if (slot >= 0) {  // one slot's ligands as ligands 0..n-1 (offsets stay absolute)
            v.ligs = d_desc.p + (size_t)slot * M;
            v.max_atoms = std::max(1, slots[slot].max_atoms);
            v.max_torsions = slots[slot].max_tors;
        }
        return v;
    }
    ~ud_stream_s() {
        if (running) {  // no further slot: the kernel drains and exits
            if (!closed && cs) {
                cudaMemcpyAsync(d_ctl.p + 1, h_counts.p + max_slots + 1, sizeof(unsigned int),
                                cudaMemcpyHostToDevice, cs);
                cudaStreamSynchronize(cs);
            }
            cudaStreamSynchronize(ks);
        }
        for (auto& e : staged)
            if (e) cudaEventDestroy(e);
        if (h_done) cudaFreeHost(h_done);
        for (cudaStream_t s : {ks, cs, ps})
            if (s) cudaStreamDestroy(s);
    }
};

extern "C" int ud_stream_create(ud_maps maps, const ud_search_params* params, const ud_stream_config* cfg,
                                ud_stream* out) {
    return guarded([&] {
        if (!maps || !params || !cfg || !out) throw Error(UD_ERR_ARG, "null argument");
        const ud_search_params& P = *params;
        if (P.exhaustiveness < 1) throw Error(UD_ERR_ARG, "exhaustiveness must be >= 1");
        // at or below every ligand's heuristic step count (70*3*(50 + N + 10*DOF)/2 >= 11655),
        // so a chain's step count does not depend on the ligands that share its slot
        if (P.max_step < 1 || P.max_step > 11655)
            throw Error(UD_ERR_ARG, "a streaming screen needs max_step in 1..11655 (--max_step)");
        if (P.num_modes < 1) throw Error(UD_ERR_ARG, "num_modes must be >= 1");
        if (P.chains_per_block < 0 || P.chains_per_block > 4)
            throw Error(UD_ERR_ARG, "chains_per_block must be 0 (default) or 1..4");
        if (P.lanes_per_chain != 0 && P.lanes_per_chain != 32)
            throw Error(UD_ERR_ARG, "a streaming screen runs one chain per warp (lanes_per_chain 0 or 32)");
        if (cfg->slot_ligands < 1 || cfg->max_slots < 1 || cfg->ring < 1 || cfg->max_atoms < 1 ||
            cfg->max_atoms > kMaxLigAtoms || cfg->max_torsions < 0 || cfg->max_torsions > kMaxLigTorsions ||
            cfg->timeout_ms < 0)
            throw Error(UD_ERR_ARG, "invalid stream configuration");
        auto st = std::make_unique<ud_stream_s>();
        st->maps = maps;
        st->params = P;
        st->E = P.exhaustiveness;
        st->M = (cfg->slot_ligands + 15) / 16 * 16;  // LigDesc blocks of whole 256-byte units
        st->max_slots = cfg->max_slots;
        st->ring = std::min(cfg->ring, cfg->max_slots);
        st->cap = P.num_modes;
        st->max_atoms = cfg->max_atoms;
        st->max_tors = cfg->max_torsions;
        st->stride = 7 + st->max_tors;
        st->ad4 = maps->desc.ad4 != 0;
        st->refined = P.refine_step > 0 && has_receptor(maps);
        SearchParams& sp = st->sp;
        sp.global_steps = P.max_step;
        sp.exhaustiveness = st->E;
        sp.seed = P.seed;
        sp.hunt_cap = 10.0f;
        sp.authentic_v = 1000.0f;
        sp.temperature = 1.2f;
        sp.mutation_amplitude = 2.0f;
        sp.lanes_per_chain = 32;
        sp.chains_per_block = P.chains_per_block;  // 0: set from the layout below
        sp.persistent = 1;
        sp.bfgs_cap = P.bfgs_cap > 0 ? P.bfgs_cap : 0;
        const size_t S = (size_t)st->max_slots, M = (size_t)st->M, E = (size_t)st->E;
        const size_t A = (size_t)st->max_atoms;
        st->atom_cap = S * aligned_elems(M * A, sizeof(AtomRec), kAtomUnit);
        st->node_cap = S * aligned_elems(M * (st->max_tors + 1), sizeof(NodeRec), kNodeUnit);
        st->grid_cap = S * aligned_elems(M * A, 4, kGridUnit);
        st->pair_cap = S * aligned_elems(M * std::max<size_t>(32, A * A / 2), 4, kPairUnit);
        cudaStream_t s0 = nullptr;
        for (cudaStream_t* s : {&st->ks, &st->cs, &st->ps})
            cuda_check(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking), "stream");
        s0 = st->cs;
        st->d_desc.alloc(S * M);
        st->d_atoms.alloc(st->atom_cap);
        st->d_nodes.alloc(st->node_cap);
        st->d_pairs.alloc(st->pair_cap);
        st->d_grid.alloc(st->grid_cap);
        if (st->ad4) {
            st->d_charge.alloc(st->atom_cap);
            st->d_coef.alloc(2 * st->pair_cap);
        }
        st->d_ctl.alloc(4);
        st->d_slot_left.alloc(S);
        st->d_slot_nlig.alloc(S);
        st->d_order.alloc(S * M);
        st->d_status.alloc(1);
        cuda_check(cudaHostAlloc((void**)&st->h_done, S * sizeof(unsigned int), cudaHostAllocMapped), "mapped memory");
        std::memset(st->h_done, 0, S * sizeof(unsigned int));
        st->h_counts.alloc(S + 2);
        for (size_t k = 0; k <= S; ++k) st->h_counts.p[k] = (unsigned int)k;
        st->h_counts.p[S + 1] = 1;
        // staging of one slot: LigDesc, order, counts, atoms, charges, nodes, pairs, coefficients, grid words
        const size_t stage = M * (sizeof(LigDesc) + 4) + 16 + M * A * (sizeof(AtomRec) + 4) +
                             M * (st->max_tors + 1) * sizeof(NodeRec) + M * std::max<size_t>(32, A * A / 2) * 12 +
                             M * A * 4 + 4096;
        for (int b = 0; b < 2; ++b) {
            st->staging[b].alloc(stage);
            cuda_check(cudaEventCreateWithFlags(&st->staged[b], cudaEventDisableTiming), "event");
            cuda_check(cudaEventRecord(st->staged[b], s0), "event");
        }
        const size_t R = (size_t)st->ring;
        st->d_poses.alloc(R * M * E * st->stride);
        st->d_results.alloc(R * M * E);
        const size_t modes = R * M * st->cap;
        st->d_scratch.alloc(modes * 3 * A);
        st->d_n_modes.alloc(R * M);
        st->d_mode_chain.alloc(modes);
        st->d_mode_lig.alloc(modes);
        st->d_mode_pose.alloc(modes * st->stride);
        st->d_mode_e.alloc(modes * 4);
        st->hp_n_modes.alloc(M);
        st->hp_mode_chain.alloc(M * st->cap);
        st->hp_mode_pose.alloc(M * st->cap * st->stride);
        st->hp_mode_e.alloc(M * st->cap * 4);
        st->hp_poses.alloc(M * E * st->stride);
        st->hp_results.alloc(M * E);
        if (st->refined) ensure_receptor(maps, s0);
        st->slots.resize(S);
        cuda_check(cudaMemsetAsync(st->d_ctl.p, 0, 4 * sizeof(unsigned int), s0), "memset");
        cuda_check(cudaMemsetAsync(st->d_status.p, 0, sizeof(int), s0), "memset");
        cuda_check(cudaStreamSynchronize(s0), "stream set-up");
        StreamView sv{};
        sv.published = st->d_ctl.p;
        sv.closed = st->d_ctl.p + 1;
        sv.next_item = st->d_ctl.p + 2;
        sv.slot_left = st->d_slot_left.p;
        sv.slot_nlig = st->d_slot_nlig.p;
        sv.order = st->d_order.p;
        unsigned int* done_dev = nullptr;
        cuda_check(cudaHostGetDevicePointer((void**)&done_dev, st->h_done, 0), "mapped pointer");
        sv.done_host = done_dev;
        sv.status = st->d_status.p;
        sv.slot_ligands = st->M;
        sv.max_slots = st->max_slots;
        sv.ring = st->ring;
        sv.timeout_ns = (unsigned long long)(cfg->timeout_ms > 0 ? cfg->timeout_ms : 60000) * 1000000ull;
        int dev = 0, n_sm = 148;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        cuda_check(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev), "device attribute");
        // one full wave of blocks; those on every reserve_every-th SM return at
        // once and leave their SM to the per-slot post-processing kernels
        cuda_check(prepare_stream_post(st->view(), st->cap, st->refined), "stream post-processing kernels");
        if (sp.chains_per_block == 0) sp.chains_per_block = default_chains_per_block(st->view(), 32, true);
        const int per_sm = stream_blocks_per_sm(st->view(), sp.chains_per_block);
        if (per_sm < 1)
            throw Error(UD_ERR_CAPACITY, "a CTA of the stream's largest ligand layout does not fit an SM");
        const int blocks = per_sm * n_sm;
        sv.reserve_every = n_sm >= 2 * kStreamReserveSms ? n_sm / kStreamReserveSms : 0;
        cuda_check(launch_search_stream(st->view(), maps_view(maps), tables_view(maps), sp, sv, st->d_poses.p,
                                        st->stride, st->d_results.p, blocks, st->ks),
                   "stream kernel");
        st->running = true;
        *out = st.release();
    });
}

extern "C" int ud_stream_push(ud_stream st, const ud_ligand* ligs, int n, int* slot) {
    return guarded([&] {
        if (!st || (n > 0 && !ligs)) throw Error(UD_ERR_ARG, "null argument");
        if (st->closed) throw Error(UD_ERR_STATE, "stream closed");
        if (n < 1 || n > st->M) throw Error(UD_ERR_ARG, "a slot holds 1.." + std::to_string(st->M) + " ligands");
        const int k = st->n_pushed;
        if (k >= st->max_slots) throw Error(UD_ERR_CAPACITY, "all slots of the stream are used");
        if (k >= st->ring && !st->slots[k - st->ring].collected)
            throw Error(UD_ERR_STATE, "slot " + std::to_string(k - st->ring) +
                                          " must be collected before its result area is reused");
        std::vector<const Ligand*> v;
        for (int i = 0; i < n; ++i) {
            if (!ligs[i]) throw Error(UD_ERR_ARG, "null ligand");
            const Ligand& L = ligs[i]->lig;
            if ((int)L.atoms.size() > st->max_atoms || L.n_torsions() > st->max_tors)
                throw Error(UD_ERR_CAPACITY, "ligand " + std::to_string(i) + " exceeds the stream's max_atoms / "
                                                                         "max_torsions");
            v.push_back(&L);
        }
        const size_t a0 = aligned_elems(st->n_atoms, sizeof(AtomRec), kAtomUnit);
        const size_t n0 = aligned_elems(st->n_nodes, sizeof(NodeRec), kNodeUnit);
        const size_t p0 = aligned_elems(st->n_pairs, 4, kPairUnit);
        const size_t g0 = aligned_elems(st->n_grid, 4, kGridUnit);
        TopologyPack tp;
        pack_topology(st->maps, v, k * st->M, a0, n0, p0, g0, tp);
        if (a0 + tp.atoms.size() > st->atom_cap || n0 + tp.nodes.size() > st->node_cap ||
            p0 + tp.pairs.size() > st->pair_cap || g0 + tp.grid_list.size() > st->grid_cap)
            throw Error(UD_ERR_CAPACITY, "the stream's arena is full");
        // stage the slot in page-locked memory (a buffer whose previous copies are done)
        PinnedBuf<unsigned char>& stg = st->staging[k & 1];
        cuda_check(cudaEventSynchronize(st->staged[k & 1]), "staging");
        size_t off = 0;
        auto put = [&](const void* src, size_t bytes) {
            off = (off + 15) & ~(size_t)15;
            if (off + bytes > stg.n) throw Error(UD_ERR_CAPACITY, "slot larger than the staging buffer");
            if (bytes) std::memcpy(stg.p + off, src, bytes);
            const size_t at = off;
            off += bytes;
            return stg.p + at;
        };
        auto copy = [&](void* dst, const void* src, size_t bytes) {
            if (bytes) cuda_check(cudaMemcpyAsync(dst, put(src, bytes), bytes, cudaMemcpyHostToDevice, st->cs), "H2D");
        };
        const unsigned int chains = (unsigned int)n * (unsigned int)st->E;
        copy(st->d_desc.p + (size_t)k * st->M, tp.desc.data(), tp.desc.size() * sizeof(LigDesc));
        copy(st->d_atoms.p + a0, tp.atoms.data(), tp.atoms.size() * sizeof(AtomRec));
        copy(st->d_nodes.p + n0, tp.nodes.data(), tp.nodes.size() * sizeof(NodeRec));
        copy(st->d_pairs.p + p0, tp.pairs.data(), tp.pairs.size() * 4);
        copy(st->d_grid.p + g0, tp.grid_list.data(), tp.grid_list.size() * 4);
        if (st->ad4) {
            copy(st->d_charge.p + a0, tp.charges.data(), tp.charges.size() * sizeof(float));
            copy(st->d_coef.p + 2 * p0, tp.coef.data(), tp.coef.size() * sizeof(float));
        }
        copy(st->d_order.p + (size_t)k * st->M, tp.order.data(), tp.order.size() * sizeof(int));
        copy(st->d_slot_nlig.p + k, &n, sizeof(int));
        copy(st->d_slot_left.p + k, &chains, sizeof(unsigned int));
        // then the published count, after every copy of the slot on the same stream
        cuda_check(cudaMemcpyAsync(st->d_ctl.p, st->h_counts.p + k + 1, sizeof(unsigned int), cudaMemcpyHostToDevice,
                                   st->cs),
                   "publish");
        cuda_check(cudaEventRecord(st->staged[k & 1], st->cs), "event");
        st->n_atoms = a0 + tp.atoms.size();
        st->n_nodes = n0 + tp.nodes.size();
        st->n_pairs = p0 + tp.pairs.size();
        st->n_grid = g0 + tp.grid_list.size();
        StreamSlot& sl = st->slots[k];
        sl.ligs = v;
        sl.max_atoms = tp.max_atoms;
        sl.max_tors = tp.max_tors;
        ++st->n_pushed;
        if (slot) *slot = k;
    });
}

static void stream_close(ud_stream st) {
    if (st->closed) return;
    cuda_check(cudaMemcpyAsync(st->d_ctl.p + 1, st->h_counts.p + st->max_slots + 1, sizeof(unsigned int),
                               cudaMemcpyHostToDevice, st->cs),
               "close");
    st->closed = true;
}

extern "C" int ud_stream_close(ud_stream st) {
    return guarded([&] {
        if (!st) throw Error(UD_ERR_ARG, "null stream");
        stream_close(st);
    });
}

// The kernel's end status once it has stopped (it stopped early when a wait
// ran out or an error ended it).
static void stream_check_kernel(ud_stream st) {
    const cudaError_t q = cudaStreamQuery(st->ks);
    if (q == cudaErrorNotReady) return;
    st->running = false;
    st->finished = true;
    cuda_check(q, "stream kernel");
    cuda_check(cudaMemcpy(&st->status, st->d_status.p, sizeof(int), cudaMemcpyDeviceToHost), "status");
}

extern "C" int ud_stream_collect(ud_stream st, int slot) {
    return guarded([&] {
        if (!st) throw Error(UD_ERR_ARG, "null stream");
        if (slot < 0 || slot >= st->n_pushed) throw Error(UD_ERR_ARG, "slot not pushed");
        StreamSlot& sl = st->slots[slot];
        if (sl.collected) return;
        // the slot's chains are done when the kernel has set its flag
        const volatile unsigned int* done = st->h_done + slot;
        while (*done == 0) {
            if (st->running) stream_check_kernel(st);
            if (!st->running) {
                if (*done) break;
                if (st->status == kStreamTimeout)
                    throw Error(UD_ERR_TIMEOUT, "the stream kernel stopped waiting for a slot to be published");
                throw Error(UD_ERR_STATE, "the stream kernel ended before slot " + std::to_string(slot) + " was done");
            }
            std::this_thread::sleep_for(std::chrono::microseconds(100));
        }
        std::atomic_thread_fence(std::memory_order_acquire);
        const int n = (int)sl.ligs.size(), E = st->E, cap = st->cap, stride = st->stride;
        const size_t r = (size_t)(slot % st->ring), M = (size_t)st->M;
        const size_t n_chain = (size_t)n * E, n_mode = (size_t)n * cap;
        float* poses = st->d_poses.p + r * M * E * stride;
        ChainResult* results = st->d_results.p + r * M * E;
        float* scratch = st->d_scratch.p + r * M * cap * 3 * st->max_atoms;
        int* n_modes = st->d_n_modes.p + r * M;
        int* mode_chain = st->d_mode_chain.p + r * M * cap;
        int* mode_lig = st->d_mode_lig.p + r * M * cap;
        float* mode_pose = st->d_mode_pose.p + r * M * cap * stride;
        float* mode_e = st->d_mode_e.p + r * M * cap * 4;
        const DeviceBatchView v = st->view(slot);
        cudaStream_t ps = st->ps;
        // launch_cluster indexes the scratch by the view's largest ligand: the slot's,
        // at most the stream's, so the stream-sized area holds it
        cuda_check(launch_cluster(v, poses, stride, results, n, E, cap, st->params.min_rmsd, scratch, n_modes,
                                  mode_chain, mode_lig, mode_pose, ps),
                   "stream clustering");
        if (st->refined) {
            DeviceReceptorView rv = st->maps->rc;
            rv.lig_bias = nullptr;
            rv.lig_bias_span = nullptr;
            cuda_check(launch_receptor(kRecRefine, v, tables_view(st->maps), rv, mode_lig, mode_pose, stride,
                                       (int)n_mode, st->params.refine_step, 0.0f, 1000.0f, nullptr, nullptr, 0,
                                       mode_e, ps),
                       "stream refinement");
        }
        auto d2h = [&](void* dst, const void* src, size_t bytes) {
            cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ps), "D2H");
        };
        d2h(st->hp_n_modes.p, n_modes, n * sizeof(int));
        d2h(st->hp_mode_chain.p, mode_chain, n_mode * sizeof(int));
        d2h(st->hp_mode_pose.p, mode_pose, n_mode * stride * sizeof(float));
        if (st->refined) d2h(st->hp_mode_e.p, mode_e, n_mode * 4 * sizeof(float));
        d2h(st->hp_results.p, results, n_chain * sizeof(ChainResult));
        d2h(st->hp_poses.p, poses, n_chain * stride * sizeof(float));
        cuda_check(cudaStreamSynchronize(ps), "stream post-processing");
        sl.results.assign(st->hp_results.p, st->hp_results.p + n_chain);
        sl.poses.assign(st->hp_poses.p, st->hp_poses.p + n_chain * stride);
        for (const ChainResult& c : sl.results) st->evals += c.evals;
        sl.post.assign(n, LigandPost{});
        parallel_for(n, [&](int l) {
            const size_t o = (size_t)l * cap;
            sl.post[l] = post_process_ligand(st->maps->sf, *sl.ligs[l], E, cap, stride, st->refined,
                                             st->hp_n_modes.p[l], st->hp_mode_chain.p + o,
                                             st->hp_mode_pose.p + o * stride, st->hp_mode_e.p + 4 * o,
                                             sl.results.data() + (size_t)l * E);
        });
        sl.collected = true;
    });
}

static const StreamSlot& collected_slot(ud_stream st, int slot, int lig) {
    if (!st) throw Error(UD_ERR_ARG, "null stream");
    if (slot < 0 || slot >= st->n_pushed || !st->slots[slot].collected) throw Error(UD_ERR_STATE, "slot not collected");
    const StreamSlot& sl = st->slots[slot];
    if (lig < 0 || lig >= (int)sl.ligs.size()) throw Error(UD_ERR_ARG, "ligand out of range");
    return sl;
}

extern "C" int ud_stream_result_count(ud_stream st, int slot, int lig, int* n_modes) {
    return guarded([&] {
        if (!n_modes) throw Error(UD_ERR_ARG, "null argument");
        *n_modes = (int)collected_slot(st, slot, lig).post[lig].modes.size();
    });
}

extern "C" int ud_stream_result_mode(ud_stream st, int slot, int lig, int k, float* pose, float energies[8]) {
    return guarded([&] {
        const auto& m = collected_slot(st, slot, lig).post[lig].modes;
        if (k < 0 || k >= (int)m.size()) throw Error(UD_ERR_ARG, "mode out of range");
        if (pose) std::copy(m[k].pose.begin(), m[k].pose.end(), pose);
        if (energies) {
            const float e[8] = {m[k].e, m[k].lb, m[k].ub, m[k].total, m[k].inter, m[k].intra, m[k].conf_indep,
                                m[k].unbound};
            std::copy(e, e + 8, energies);
        }
    });
}

extern "C" int ud_stream_result_write(ud_stream st, int slot, int lig, int format, char* buf, size_t cap,
                                      size_t* len) {
    return guarded([&] {
        const StreamSlot& sl = collected_slot(st, slot, lig);
        if (format != 0 && format != 1) throw Error(UD_ERR_ARG, "format must be 0 (PDBQT) or 1 (SDF)");
        const std::string t = render_modes(*sl.ligs[lig], sl.post[lig], st->params.num_modes,
                                           st->params.energy_range, st->ad4, format);
        if (len) *len = t.size();
        if (buf && cap > 0) {
            const size_t n = std::min(cap - 1, t.size());
            std::memcpy(buf, t.data(), n);
            buf[n] = 0;
        }
    });
}

extern "C" int ud_stream_chains(ud_stream st, int slot, float* poses, int pose_stride, float* e, int* evals) {
    return guarded([&] {
        const StreamSlot& sl = collected_slot(st, slot, 0);
        const size_t n_chain = sl.results.size();
        if (poses) {
            if (pose_stride < 7 + st->max_tors) throw Error(UD_ERR_ARG, "pose_stride smaller than 7 + max_torsions");
            for (size_t i = 0; i < n_chain; ++i)
                std::copy(sl.poses.begin() + i * st->stride, sl.poses.begin() + (i + 1) * st->stride,
                          poses + i * pose_stride);
        }
        for (size_t i = 0; i < n_chain; ++i) {
            if (e) e[i] = sl.results[i].e;
            if (evals) evals[i] = sl.results[i].evals;
        }
    });
}

extern "C" int ud_stream_finish(ud_stream st, long long* evals) {
    return guarded([&] {
        if (!st) throw Error(UD_ERR_ARG, "null stream");
        if (st->running) {
            cuda_check(cudaStreamSynchronize(st->ks), "stream kernel");
            stream_check_kernel(st);
        }
        if (evals) *evals = st->evals;
        if (st->status == kStreamTimeout)
            throw Error(UD_ERR_TIMEOUT, "the stream kernel stopped waiting for a slot to be published");
    });
}

extern "C" int ud_stream_destroy(ud_stream st) {
    delete st;
    return UD_OK;
}
