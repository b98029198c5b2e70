// unidock -- command-line host of the B200 docking engine.
//
// Drop-in for the reference CLI's docking paths (unidock/src/main/main.cpp:
// options :421-575, search_mode presets :644-661, checks :705-760, GPU batch
// flow :904-1070): same option names, the same output file names
// (utils.cpp default_output / default_score_output) and the same PDBQT result
// format.  Everything goes through the C ABI of libunidock_b200.
//
// Batch mode keeps two batches in flight on two CUDA streams: while the GPU
// searches one batch, the host parses and uploads the next one and
// post-processes and writes the previous one.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <vector>

#include "../../../include/unidock_b200.h"

namespace {

// ---------------------------------------------------------------- options
struct OptSpec {
    const char* name;
    int kind;  // 0 = value, 1 = switch, 2 = multi-token values
    const char* help;
    const char* group;
};

const OptSpec kOptions[] = {
    {"receptor", 0, "rigid part of the receptor (PDBQT)", "Input"},
    {"flex", 0, "flexible side chains (not supported by this engine)", "Input"},
    {"ligand", 2, "ligand (PDBQT or SDF)", "Input"},
    {"ligand_index", 0, "file containing paths to ligands (PDBQT or SDF)", "Input"},
    {"paired_batch_size", 0, "If > 0, uses batching for one-ligand-one-protein docking, with json config in "
                             "ligand_index following paired_batching.schema.json", "Input"},
    {"batch", 2, "batch ligand (PDBQT)", "Input"},
    {"gpu_batch", 2, "gpu batch ligand (PDBQT or SDF)", "Input"},
    {"scoring", 0, "scoring function (ad4, vina or vinardo)", "Input"},
    {"maps", 0, "affinity maps for the autodock4.2 (ad4) or vina scoring function (AutoGrid .map files "
                "<prefix>.<type>.map)", "Search space"},
    {"center_x", 0, "X coordinate of the center (Angstrom)", "Search space"},
    {"center_y", 0, "Y coordinate of the center (Angstrom)", "Search space"},
    {"center_z", 0, "Z coordinate of the center (Angstrom)", "Search space"},
    {"size_x", 0, "size in the X dimension (Angstrom)", "Search space"},
    {"size_y", 0, "size in the Y dimension (Angstrom)", "Search space"},
    {"size_z", 0, "size in the Z dimension (Angstrom)", "Search space"},
    {"autobox", 1, "set maps dimensions based on input ligand(s) (for --score_only and --local_only)",
     "Search space"},
    {"out", 0, "output models (PDBQT), the default is chosen based on the ligand file name", "Output"},
    {"dir", 0, "output directory for batch mode", "Output"},
    {"write_maps", 0, "output filename (directory + prefix name) for maps", "Output"},
    {"device_id", 0, "GPU device id to use (default 0)", "Advanced"},
    {"score_only", 1, "score only - search space can be omitted", "Advanced"},
    {"score_file", 0, "score only output file in batch mode, with 'score_only' option", "Advanced"},
    {"local_only", 1, "do local search only", "Advanced"},
    {"no_refine", 1, "when --receptor is provided, do not use explicit receptor atoms (instead of precalculated "
                     "grids) for: (1) local optimization and scoring after docking, (2) --local_only and "
                     "--score_only", "Advanced"},
    {"force_even_voxels", 1, "calculated grid maps will have an even number of voxels in each dimension",
     "Advanced"},
    {"randomize_only", 1, "randomize input (not supported by this engine)", "Advanced"},
    {"weight_gauss1", 0, "gauss_1 weight", "Advanced"},
    {"weight_gauss2", 0, "gauss_2 weight", "Advanced"},
    {"weight_repulsion", 0, "repulsion weight", "Advanced"},
    {"weight_hydrophobic", 0, "hydrophobic weight", "Advanced"},
    {"weight_hydrogen", 0, "Hydrogen bond weight", "Advanced"},
    {"weight_rot", 0, "N_rot weight", "Advanced"},
    {"weight_vinardo_gauss1", 0, "Vinardo gauss_1 weight", "Advanced"},
    {"weight_vinardo_repulsion", 0, "Vinardo repulsion weight", "Advanced"},
    {"weight_vinardo_hydrophobic", 0, "Vinardo hydrophobic weight", "Advanced"},
    {"weight_vinardo_hydrogen", 0, "Vinardo Hydrogen bond weight", "Advanced"},
    {"weight_vinardo_rot", 0, "Vinardo N_rot weight", "Advanced"},
    {"weight_ad4_vdw", 0, "ad4_vdw weight", "Advanced"},
    {"weight_ad4_hb", 0, "ad4_hb weight", "Advanced"},
    {"weight_ad4_elec", 0, "ad4_elec weight", "Advanced"},
    {"weight_ad4_dsolv", 0, "ad4_dsolv weight", "Advanced"},
    {"weight_ad4_rot", 0, "ad4_rot weight", "Advanced"},
    {"weight_glue", 0, "macrocycle glue weight", "Advanced"},
    {"bias", 0, "bias configuration file name, content similar to BPF in AutoDock-bias", "Advanced"},
    {"multi_bias", 1, "add ligand bias {ligand_name}.bpf for every input ligand, content similar to BPF in "
                      "AutoDock-bias", "Advanced"},
    {"keep_nonpolar_H", 1, "keep non polar H in sdf", "Advanced"},
    {"cpu", 0, "the number of CPUs to use for parsing and post-processing (0 = all)", "Misc"},
    {"seed", 0, "explicit random seed", "Misc"},
    {"exhaustiveness", 0, "exhaustiveness of the global search (roughly proportional to time): 1+", "Misc"},
    {"max_evals", 0, "number of evaluations in each MC run (accepted; the step count governs)", "Misc"},
    {"num_modes", 0, "maximum number of binding modes to generate", "Misc"},
    {"min_rmsd", 0, "minimum RMSD between output poses", "Misc"},
    {"energy_range", 0, "maximum energy difference between the best binding mode and the worst one displayed "
                        "(kcal/mol)", "Misc"},
    {"spacing", 0, "grid spacing (Angstrom)", "Misc"},
    {"verbosity", 0, "verbosity (0=no output, 1=normal, 2=verbose)", "Misc"},
    {"max_step", 0, "maximum number of steps in each MC run (if zero, the number of MC steps is based on "
                    "heuristics)", "Misc"},
    {"refine_step", 0, "number of steps in refinement, default=3", "Misc"},
    {"max_gpu_memory", 0, "maximum gpu memory to use in MiB (default=0, use the available memory)", "Misc"},
    {"search_mode", 0, "search mode of vina (fast, balance, detail)", "Misc"},
    {"batch_size", 0, "ligands per GPU batch (default 4096)", "Misc"},
    {"autotune", 1, "pick chains per CTA and the BFGS cap per batch with the autotuner", "Misc"},
    {"config", 0, "the above options can be put here", "Configuration file"},
    {"help", 1, "display usage summary", "Information"},
    {"help_advanced", 1, "display usage summary with advanced options", "Information"},
    {"version", 1, "display program version", "Information"},
};

const OptSpec* find_opt(const std::string& n) {
    for (const auto& o : kOptions)
        if (n == o.name) return &o;
    return nullptr;
}

struct Options {
    std::map<std::string, std::vector<std::string>> v;
    bool has(const std::string& k) const { return v.count(k) > 0; }
    std::string str(const std::string& k, const std::string& d = "") const {
        auto it = v.find(k);
        return it == v.end() || it->second.empty() ? d : it->second.back();
    }
    double num(const std::string& k, double d) const {
        auto it = v.find(k);
        if (it == v.end() || it->second.empty()) return d;
        char* end = nullptr;
        double x = std::strtod(it->second.back().c_str(), &end);
        if (!end || *end) throw std::runtime_error("invalid number for --" + k + ": " + it->second.back());
        return x;
    }
    std::vector<std::string> list(const std::string& k) const {
        auto it = v.find(k);
        return it == v.end() ? std::vector<std::string>{} : it->second;
    }
};

void add_value(Options& o, const OptSpec* s, const std::string& val) {
    if (s->kind == 1) {  // switches: "0" / "false" turn them off (config files)
        if (val == "0" || val == "false")
            o.v.erase(s->name);
        else
            o.v[s->name] = {"1"};
    } else if (s->kind == 2) {
        o.v[s->name].push_back(val);
    } else {
        o.v[s->name] = {val};
    }
}

void parse_args(int argc, char** argv, Options& o) {
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a.rfind("--", 0) != 0) throw std::runtime_error("unexpected argument: " + a);
        std::string key = a.substr(2), val;
        bool inline_val = false;
        if (auto eq = key.find('='); eq != std::string::npos) {
            val = key.substr(eq + 1);
            key = key.substr(0, eq);
            inline_val = true;
        }
        const OptSpec* s = find_opt(key);
        if (!s) throw std::runtime_error("unrecognised option '--" + key + "'");
        if (s->kind == 1) {
            add_value(o, s, inline_val ? val : "1");
        } else if (inline_val) {
            add_value(o, s, val);
        } else if (s->kind == 2) {
            int n = 0;
            while (i + 1 < argc && std::strncmp(argv[i + 1], "--", 2) != 0) {
                add_value(o, s, argv[++i]);
                ++n;
            }
            if (!n) throw std::runtime_error("the required argument for option '--" + key + "' is missing");
        } else {
            if (i + 1 >= argc) throw std::runtime_error("the required argument for option '--" + key + "' is missing");
            add_value(o, s, argv[++i]);
        }
    }
}

// "name = value" lines; command-line values take precedence
void parse_config(const std::string& path, Options& o) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("could not open config file " + path);
    Options c;
    std::string line;
    while (std::getline(f, line)) {
        if (auto h = line.find('#'); h != std::string::npos) line.resize(h);
        auto eq = line.find('=');
        if (eq == std::string::npos) continue;
        auto trim = [](std::string s) {
            s.erase(0, s.find_first_not_of(" \t\r"));
            s.erase(s.find_last_not_of(" \t\r") + 1);
            return s;
        };
        std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
        const OptSpec* s = find_opt(k);
        if (!s) throw std::runtime_error("unrecognised option '" + k + "' in " + path);
        add_value(c, s, v);
    }
    for (auto& kv : c.v)
        if (!o.has(kv.first)) o.v[kv.first] = kv.second;
}

void usage(bool advanced) {
    std::cout << "Usage: unidock --receptor R.pdbqt (--ligand L.pdbqt | --gpu_batch L1 L2 ... | --ligand_index F) "
                 "--center_x X --center_y Y --center_z Z --size_x SX --size_y SY --size_z SZ [--dir D] [options]\n";
    std::string group;
    for (const auto& o : kOptions) {
        if (!advanced && std::strcmp(o.group, "Advanced") == 0) continue;
        if (group != o.group) {
            group = o.group;
            std::cout << "\n" << group << ":\n";
        }
        std::cout << "  --" << std::left << std::setw(28) << o.name << o.help << "\n";
    }
}

// ---------------------------------------------------------------- files
std::string read_file(const std::string& p) {
    std::ifstream f(p, std::ios::binary);
    if (!f) throw std::runtime_error("could not open \"" + p + "\" for reading");
    std::ostringstream s;
    s << f.rdbuf();
    return s.str();
}

bool ends_with(const std::string& s, const std::string& t) {
    return s.size() >= t.size() && s.compare(s.size() - t.size(), t.size(), t) == 0;
}

std::string get_filename(const std::string& s) {
    auto i = s.rfind('/');
    return i == std::string::npos ? s : s.substr(i + 1);
}

// utils.cpp default_output / default_score_output
std::string strip_ext(const std::string& n) {
    if (ends_with(n, ".pdbqt")) return n.substr(0, n.size() - 6);
    if (ends_with(n, ".sdf")) return n.substr(0, n.size() - 4);
    return n;
}
std::string default_output(const std::string& name) {
    return strip_ext(name) + (ends_with(name, ".sdf") ? "_out.sdf" : "_out.pdbqt");
}
std::string default_output(const std::string& name, const std::string& dir) {
    return dir + "/" + default_output(name);
}
std::string default_score_output(const std::string& name) { return strip_ext(name) + "_score.txt"; }

bool file_exists(const std::string& p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

bool is_directory(const std::string& p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

void check(int rc, const char* what) {
    if (rc != UD_OK) throw std::runtime_error(std::string(what) + ": " + ud_last_error());
}

template <class F> void parallel_for(int n, int threads, F&& body) {
    if (n <= 0) return;
    threads = std::max(1, std::min(threads, n));
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&] {
            for (int i; (i = next.fetch_add(1)) < n;) body(i);
        });
    for (auto& th : pool) th.join();
}

struct ParsedLigand {
    std::string path;
    ud_ligand h = nullptr;
};

// parse_ligand_from_file_no_failure: unreadable or malformed ligands are
// reported and skipped
std::vector<ParsedLigand> parse_ligands(const std::vector<std::string>& paths, int threads, int verbosity) {
    std::vector<ParsedLigand> out(paths.size());
    parallel_for((int)paths.size(), threads, [&](int i) {
        out[i].path = paths[i];
        try {
            std::string t = read_file(paths[i]);
            // by file name, as parse_ligand_from_file_no_failure; hydrogens are
            // always kept (--keep_nonpolar_H is a switch that defaults to on)
            const int rc = ends_with(paths[i], ".sdf") ? ud_ligand_parse_sdf(t.data(), t.size(), 1, &out[i].h)
                                                       : ud_ligand_parse(t.data(), t.size(), &out[i].h);
            if (rc != UD_OK) {
                out[i].h = nullptr;
                throw std::runtime_error(ud_last_error());
            }
        } catch (const std::exception& e) {
            if (verbosity > 0) std::cerr << "WARNING: skipping ligand " << paths[i] << ": " << e.what() << "\n";
        }
    });
    std::vector<ParsedLigand> ok;
    for (auto& p : out)
        if (p.h) ok.push_back(p);
    return ok;
}

void print_energies(std::ostream& os, const float* e) {
    os << std::fixed << std::setprecision(3);
    os << "Estimated Free Energy of Binding   : " << e[0] << " (kcal/mol) [=(1)+(2)+(3)+(4)]\n";
    os << "(1) Final Intermolecular Energy    : " << e[1] + e[2] << " (kcal/mol)\n";
    os << "    Ligand - Receptor              : " << e[1] << " (kcal/mol)\n";
    os << "    Ligand - Flex side chains      : " << e[2] << " (kcal/mol)\n";
    os << "(2) Final Total Internal Energy    : " << e[3] + e[4] + e[5] << " (kcal/mol)\n";
    os << "    Ligand                         : " << e[5] << " (kcal/mol)\n";
    os << "    Flex   - Receptor              : " << e[3] << " (kcal/mol)\n";
    os << "    Flex   - Flex side chains      : " << e[4] << " (kcal/mol)\n";
    os << "(3) Torsional Free Energy          : " << e[6] << " (kcal/mol)\n";
    os << "(4) Unbound System's Energy        : " << e[7] << " (kcal/mol)\n";
}

void print_modes(ud_batch b, int lig, int num_modes, double energy_range) {
    int n = 0;
    check(ud_result_count(b, lig, &n), "results");
    std::cout << "mode |   affinity | dist from best mode\n"
                 "     | (kcal/mol) | rmsd l.b.| rmsd u.b.\n"
                 "-----+------------+----------+----------\n";
    float best = 0;
    for (int k = 0; k < n && k < num_modes; ++k) {
        std::vector<float> pose(7 + 64);
        float en[8];
        check(ud_result_mode(b, lig, k, pose.data(), en), "mode");
        if (k == 0) best = en[0];
        if (en[0] > best + energy_range) break;
        std::cout << std::setw(4) << k + 1 << "    " << std::setw(9) << std::fixed << std::setprecision(3) << en[0]
                  << "  " << std::setw(9) << std::setprecision(3) << en[1] << "  " << std::setw(9) << en[2] << "\n";
    }
}

struct Setup {
    int sf = UD_SF_VINA;
    std::vector<float> weights;
    float center[3] = {0, 0, 0}, size[3] = {0, 0, 0};
    float spacing = 0.375f;
    ud_search_params params{};
    int verbosity = 1;
    int threads = 1;
    bool autotune = false;
    // scores after docking, --score_only and --local_only against the receptor
    // atoms (the reference unless --no_refine; Vina / Vinardo with --receptor)
    bool receptor_scoring = false;
    bool multi_bias = false;  // --multi_bias: each batch ligand's own {name}.bpf
};

// get_biasname (utils.cpp:103-111): the ligand file name without .pdbqt / .sdf, plus .bpf
std::string bias_name(const std::string& path) {
    std::string t = path;
    if (t.size() >= 6 && t.compare(t.size() - 6, 6, ".pdbqt") == 0) t.resize(t.size() - 6);
    else if (t.size() >= 4 && t.compare(t.size() - 4, 4, ".sdf") == 0) t.resize(t.size() - 4);
    return t + ".bpf";
}

// --score_only / --local_only energy vector of one pose (Vina::score, vina.cpp:1168-1243).
void score_pose(const Setup& S, ud_batch b, std::vector<float>& pose, float* en) {
    int lig = 0;
    if (S.receptor_scoring)
        check(ud_score_terms_receptor(b, &lig, pose.data(), 1, (int)pose.size(), en, nullptr), "score");
    else
        check(ud_score_terms(b, &lig, pose.data(), 1, (int)pose.size(), en, nullptr), "score");
}

// Vina::optimize (vina.cpp:1385-1428): up to five rounds of BFGS on the maps at
// curl cap 1000, until the heavy atoms are inside the box (cache::is_in_grid,
// margin 1e-4).
void local_optimize(ud_maps maps, ud_batch b, ud_ligand h, std::vector<float>& pose) {
    int counts[8];
    check(ud_ligand_counts(h, counts), "ligand");
    const int n = counts[0];
    std::vector<int> el(n);
    check(ud_ligand_export(h, nullptr, nullptr, nullptr, nullptr, el.data(), nullptr, nullptr, nullptr, nullptr,
                           nullptr, nullptr, nullptr, nullptr),
          "ligand");
    int dims[3], n_maps = 0;
    float init[3], factor[3];
    check(ud_maps_info(maps, dims, init, factor, &n_maps), "maps");
    std::vector<float> xyz(3 * (size_t)n);
    const float margin = 1e-4f;
    for (int round = 0; round < 5; ++round) {
        int lig = 0, ev = 0;
        float e = 0;
        check(ud_optimize(b, &lig, pose.data(), 1, (int)pose.size(), 0, 1000.0f, &e, &ev, nullptr), "optimize");
        check(ud_ligand_coords(h, pose.data(), xyz.data()), "coords");
        bool inside = true;
        for (int a = 0; a < n && inside; ++a) {
            if (el[a] == 0) continue;  // hydrogen
            for (int k = 0; k < 3; ++k) {
                const float end = init[k] + (dims[k] - 1) / factor[k];
                if (xyz[3 * a + k] < init[k] - margin || xyz[3 * a + k] > end + margin) inside = false;
            }
        }
        if (inside) break;
    }
}

// Maps from the receptor: Vina / Vinardo maps, or AD4 maps (types and charges
// from the receptor PDBQT) in place of the external autogrid4 step.
ud_maps build_maps(const Setup& S, const std::string& receptor) {
    std::string text = read_file(receptor);
    int n = 0;
    check(ud_receptor_parse_ex(text.data(), text.size(), nullptr, nullptr, nullptr, nullptr, 0, &n), "receptor");
    std::vector<float> xyz(3 * (size_t)n), q(n);
    std::vector<int> xs(n), ad(n);
    check(ud_receptor_parse_ex(text.data(), text.size(), xyz.data(), xs.data(), ad.data(), q.data(), n, &n),
          "receptor");
    ud_maps maps = nullptr;
    if (S.sf == UD_SF_AD4) {
        check(ud_maps_create_ad4(S.weights.data(), (int)S.weights.size(), xyz.data(), ad.data(), q.data(), n,
                                 S.center, S.size, S.spacing, nullptr, 0, nullptr, &maps),
              "AD4 grid maps");
        return maps;
    }
    check(ud_maps_create(S.sf, S.weights.data(), (int)S.weights.size(), xyz.data(), xs.data(), n, S.center, S.size,
                         S.spacing, nullptr, 0, nullptr, &maps),
          "grid maps");
    return maps;
}

void write_text(const std::string& path, const std::string& text) {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("could not open \"" + path + "\" for writing");
    f << text;
}

std::string result_text(ud_batch b, int lig, int format) {
    size_t len = 0;
    check(ud_result_write(b, lig, format, nullptr, 0, &len), "write");
    std::string s(len + 1, '\0');
    check(ud_result_write(b, lig, format, &s[0], s.size(), &len), "write");
    s.resize(len);
    return s;
}

// ---------------------------------------------------------------- batch mode
// Ligands of a batch kept within `budget` device bytes (ud_batch_device_bytes;
// 0 = no limit): the largest leading count that fits, the rest returned for
// the next batch, as the reference packs batches until its predicted peak
// memory reaches --max_gpu_memory (main.cpp:139-206, 993-1070).
std::vector<ParsedLigand> fit_budget(const Setup& S, std::vector<ParsedLigand>& ligs, size_t budget) {
    std::vector<ParsedLigand> rest;
    if (budget == 0 || ligs.empty()) return rest;
    auto bytes_of = [&](size_t n) {
        std::vector<ud_ligand> hs;
        for (size_t i = 0; i < n; ++i) hs.push_back(ligs[i].h);
        size_t b = 0;
        check(ud_batch_device_bytes(hs.data(), (int)n, S.sf, &S.params, &b), "memory estimate");
        return b;
    };
    if (bytes_of(1) > budget)
        throw std::runtime_error("--max_gpu_memory leaves too little device memory for one ligand of " + ligs[0].path);
    size_t n = ligs.size();
    for (size_t b; n > 1 && (b = bytes_of(n)) > budget;)
        n = std::max<size_t>(1, std::min(n - 1, (size_t)((double)n * (double)budget / (double)b)));
    rest.assign(ligs.begin() + n, ligs.end());
    ligs.resize(n);
    return rest;
}

void run_batches(const Setup& S, ud_maps maps, const std::vector<std::string>& paths, const std::string& dir,
                 int batch_size, size_t slot_budget) {
    struct Slot {
        std::vector<ParsedLigand> ligs;
        ud_batch b = nullptr;
        cudaStream_t s = nullptr;
        std::chrono::steady_clock::time_point t0;
        int id = 0;
    };
    Slot slots[2];
    for (auto& sl : slots)
        if (cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking) != cudaSuccess)
            throw std::runtime_error("could not create a CUDA stream");
    // end of each slot's last launched batch on the device: the other slot's
    // next search is queued behind it, so that the persistent search of the
    // next batch does not take the SMs from this batch's clustering and
    // refinement kernels
    cudaEvent_t slot_done[2];
    for (auto& e : slot_done)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            throw std::runtime_error("could not create a CUDA event");
    bool has_done[2] = {false, false};
    size_t next = 0;
    int batch_id = 0, done = 0;
    std::vector<ParsedLigand> carry;  // parsed, but over the previous batch's memory budget
    auto start_batch = [&](Slot& sl) -> bool {
        sl.ligs.swap(carry);
        carry.clear();
        while (sl.ligs.size() < (size_t)batch_size && next < paths.size()) {
            const size_t take = std::min(paths.size() - next, (size_t)batch_size - sl.ligs.size());
            std::vector<std::string> chunk(paths.begin() + next, paths.begin() + next + take);
            next += take;
            for (auto& p : parse_ligands(chunk, S.threads, S.verbosity)) sl.ligs.push_back(p);
        }
        if (sl.ligs.empty()) return false;
        carry = fit_budget(S, sl.ligs, slot_budget);
        std::vector<ud_ligand> hs;
        for (auto& p : sl.ligs) hs.push_back(p.h);
        // each slot keeps its batch handle: reused, it allocates (and frees,
        // which would wait for the other slot's search) nothing once warm
        if (sl.b)
            check(ud_batch_reset(sl.b, hs.data(), (int)hs.size(), sl.s), "batch");
        else
            check(ud_batch_create(maps, hs.data(), (int)hs.size(), sl.s, &sl.b), "batch");
        if (S.multi_bias)  // each ligand's {name}.bpf (main.cpp:255-265, utils.cpp:103-111)
            for (size_t i = 0; i < sl.ligs.size(); ++i) {
                const std::string bpf = read_file(bias_name(sl.ligs[i].path));
                check(ud_batch_set_bias(sl.b, (int)i, bpf.data(), bpf.size()), "bias");
            }
        sl.id = ++batch_id;
        sl.t0 = std::chrono::steady_clock::now();
        ud_search_params p = S.params;
        if (S.autotune) {
            ud_tune_result r;
            check(ud_autotune(sl.b, &p, &r, sl.s), "autotune");
            p.chains_per_block = 0;
            p.lanes_per_chain = 0;
            p.bfgs_cap = -1;
            if (S.verbosity > 1)
                std::cout << "Batch " << sl.id << " autotuned: " << r.chains_per_block << " warps/CTA, "
                          << r.lanes_per_chain << " lanes/chain, BFGS cap " << r.bfgs_cap << "\n";
        }
        if (S.verbosity > 0) std::cout << "Batch " << sl.id << " size: " << sl.ligs.size() << std::endl;
        const int me = (int)(&sl - slots), other = me ^ 1;
        if (has_done[other]) cudaStreamWaitEvent(sl.s, slot_done[other], 0);
        check(ud_search_launch(sl.b, &p, sl.s), "search");
        cudaEventRecord(slot_done[me], sl.s);
        has_done[me] = true;
        return true;
    };
    auto finish_batch = [&](Slot& sl) {
        check(ud_search_collect(sl.b, sl.s), "search");
        for (size_t i = 0; i < sl.ligs.size(); ++i) {
            int n = 0;
            check(ud_result_count(sl.b, (int)i, &n), "results");
            if (n == 0) {
                std::cerr << "WARNING: Could not find any poses. No poses were written.\n";
                continue;
            }
            const std::string name = default_output(get_filename(sl.ligs[i].path), dir);
            write_text(name, result_text(sl.b, (int)i, ends_with(name, ".sdf") ? 1 : 0));
        }
        done += (int)sl.ligs.size();
        if (S.verbosity > 0)
            std::cout << "Batch " << sl.id << " running time: "
                      << std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() -
                                                                               sl.t0)
                             .count()
                      << "ms" << std::endl;
        for (auto& p : sl.ligs) ud_ligand_destroy(p.h);
        sl.ligs.clear();
    };
    bool live[2] = {start_batch(slots[0]), false};
    int cur = 0;
    while (live[cur]) {
        const int other = cur ^ 1;
        live[other] = start_batch(slots[other]);  // next batch queued behind this one
        finish_batch(slots[cur]);
        live[cur] = false;
        cur = other;
    }
    for (auto& sl : slots)
        if (sl.b) ud_batch_destroy(sl.b);
    for (auto& e : slot_done) cudaEventDestroy(e);
    for (auto& sl : slots) cudaStreamDestroy(sl.s);
    if (S.verbosity > 0) std::cout << "Docked ligands: " << done << std::endl;
}

// single ligand: search, local optimisation or scoring of one input pose
void run_single(const Setup& S, ud_maps maps, const std::string& path, const std::string& out_name, bool score_only,
                bool local_only) {
    auto ligs = parse_ligands({path}, 1, 2);
    if (ligs.empty()) throw std::runtime_error("could not parse ligand " + path);
    ud_ligand h = ligs[0].h;
    ud_batch b = nullptr;
    check(ud_batch_create(maps, &h, 1, nullptr, &b), "batch");
    int counts[8];
    check(ud_ligand_counts(h, counts), "ligand");
    const int stride = 7 + counts[2];
    std::vector<float> pose(stride);
    check(ud_ligand_initial_pose(h, pose.data()), "ligand");
    float en[8];
    if (score_only || local_only) {
        if (local_only) local_optimize(maps, b, h, pose);
        score_pose(S, b, pose, en);
        print_energies(std::cout, en);
        if (score_only) {
            std::ostringstream f;
            f << "REMARK " << get_filename(path) << ' ' << std::fixed << std::setprecision(3) << en[0]
              << " (kcal/mol)\n";
            print_energies(f, en);
            write_text(default_score_output(path), f.str());
        } else {
            // Vina::write_pose with no remark: the input structure with the
            // optimised coordinates (vina.cpp:1018-1030); an SDF ligand keeps
            // SDF coordinate columns
            size_t len = 0;
            check(ud_ligand_write(h, pose.data(), nullptr, 0, &len), "write");
            std::string o(len + 1, '\0');
            check(ud_ligand_write(h, pose.data(), &o[0], o.size(), &len), "write");
            o.resize(len);
            write_text(out_name, o);
        }
    } else {
        check(ud_search(b, &S.params, nullptr), "search");
        if (S.verbosity > 0) print_modes(b, 0, S.params.num_modes, S.params.energy_range);
        write_text(out_name, result_text(b, 0, ends_with(out_name, ".sdf") ? 1 : 0));
    }
    ud_batch_destroy(b);
    ud_ligand_destroy(h);
}

// ---------------------------------------------------------------- paired batches
// A small JSON reader for the paired-batch configuration: objects, strings,
// numbers, true/false/null and arrays (only objects, strings and numbers are
// used).  Object members keep their file order, as the reference's
// property tree does.
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    double num = 0;
    std::string str;
    std::vector<Json> items;                           // array elements
    std::vector<std::pair<std::string, Json>> members;  // object members in order
    const Json* get(const std::string& k) const {
        for (auto& m : members)
            if (m.first == k) return &m.second;
        return nullptr;
    }
};

struct JsonReader {
    const std::string& t;
    size_t i = 0;
    explicit JsonReader(const std::string& text) : t(text) {}
    [[noreturn]] void fail(const std::string& what) {
        throw std::runtime_error("JSON: " + what + " at offset " + std::to_string(i));
    }
    void ws() {
        while (i < t.size() && std::isspace((unsigned char)t[i])) ++i;
    }
    std::string string() {
        if (t[i] != '"') fail("expected a string");
        std::string out;
        for (++i; i < t.size() && t[i] != '"'; ++i) {
            if (t[i] != '\\') {
                out += t[i];
                continue;
            }
            if (++i >= t.size()) break;
            const char e = t[i];
            if (e == 'n') out += '\n';
            else if (e == 't') out += '\t';
            else if (e == 'r') out += '\r';
            else if (e == 'b') out += '\b';
            else if (e == 'f') out += '\f';
            else if (e == 'u') {
                if (i + 4 >= t.size()) fail("bad escape");
                const unsigned cp = (unsigned)std::stoul(t.substr(i + 1, 4), nullptr, 16);
                i += 4;
                if (cp < 0x80) out += (char)cp;  // paths and numbers only need ASCII
                else fail("non-ASCII escape");
            } else out += e;
        }
        if (i >= t.size()) fail("unterminated string");
        ++i;
        return out;
    }
    Json value() {
        ws();
        if (i >= t.size()) fail("unexpected end");
        Json v;
        const char c = t[i];
        if (c == '{') {
            v.kind = Json::Object;
            ++i;
            ws();
            if (i < t.size() && t[i] == '}') { ++i; return v; }
            for (;;) {
                ws();
                std::string k = string();
                ws();
                if (i >= t.size() || t[i] != ':') fail("expected ':'");
                ++i;
                v.members.emplace_back(k, value());
                ws();
                if (i < t.size() && t[i] == ',') { ++i; continue; }
                if (i < t.size() && t[i] == '}') { ++i; return v; }
                fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = Json::Array;
            ++i;
            ws();
            if (i < t.size() && t[i] == ']') { ++i; return v; }
            for (;;) {
                v.items.push_back(value());
                ws();
                if (i < t.size() && t[i] == ',') { ++i; continue; }
                if (i < t.size() && t[i] == ']') { ++i; return v; }
                fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = Json::String;
            v.str = string();
            return v;
        }
        if (t.compare(i, 4, "true") == 0) { v.kind = Json::Bool; v.num = 1; i += 4; return v; }
        if (t.compare(i, 5, "false") == 0) { v.kind = Json::Bool; i += 5; return v; }
        if (t.compare(i, 4, "null") == 0) { i += 4; return v; }
        size_t used = 0;
        try {
            v.num = std::stod(t.substr(i, 64), &used);
        } catch (...) {
            fail("unexpected character");
        }
        v.kind = Json::Number;
        i += used;
        return v;
    }
};

Json read_json(const std::string& path) {
    const std::string text = read_file(path);
    JsonReader r(text);
    Json v = r.value();
    r.ws();
    if (r.i != text.size()) r.fail("trailing characters");
    return v;
}

struct PairedComplex {
    std::string protein, ligand;
    float center[3], size[3];
};

// One complex's box (simulation_container.h fill_config_from_json /
// fill_config): a .json ligand config needs center_x/y/z and size_x/y/z; any
// other file holds "key=value" lines, the centre first, then optionally the
// size.  The box given on the command line is the default size.
bool read_ligand_config(const std::string& path, const float* box, PairedComplex& c) {
    for (int k = 0; k < 3; ++k) c.size[k] = box[k];
    if (ends_with(path, ".json")) {
        Json v = read_json(path);
        const char* keys[6] = {"center_x", "center_y", "center_z", "size_x", "size_y", "size_z"};
        float vals[6];
        for (int k = 0; k < 6; ++k) {
            const Json* f = v.get(keys[k]);
            if (!f || f->kind != Json::Number) {
                std::cout << "Error parsing config json " << path << "\n";
                return false;
            }
            vals[k] = (float)f->num;
        }
        for (int k = 0; k < 3; ++k) {
            c.center[k] = vals[k];
            c.size[k] = vals[3 + k];
        }
        return true;
    }
    std::ifstream in(path);
    if (!in) return false;
    std::vector<double> vals;
    for (std::string line; std::getline(in, line);) {
        line.erase(std::remove(line.begin(), line.end(), '\r'), line.end());
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        vals.push_back(std::stod(line.substr(eq + 1)));
    }
    if (vals.size() < 3) return false;
    for (int k = 0; k < 3; ++k) c.center[k] = (float)vals[k];
    if (vals.size() >= 6)
        for (int k = 0; k < 3; ++k) c.size[k] = (float)vals[3 + k];
    return true;
}

// Paired batches (simulation_container.h, vina_cuda_worker.h): every complex
// of the configuration is its own receptor, box and ligand.  The reference
// runs one host thread and CUDA stream per complex; here each batch of
// complexes is set up (maps, ligand, batch) and all its searches are queued on
// a pool of streams, so the GPU runs them side by side, then collected.
// Per complex: <dir>/<ligand>_out.pdbqt and <dir>/<ligand>_score.txt with the
// best affinity.  As the reference's worker: Vina weights, min_rmsd 0, energy
// range 3, the command line's exhaustiveness, max_step, num_modes,
// refine_step and seed.
int run_paired(const Setup& S0, const std::string& config, const std::string& dir, int batch_size, const float* box,
               bool local_only) {
    if (local_only) throw std::runtime_error("--local_only with --paired_batch_size is not supported by this engine");
    Setup S = S0;
    S.sf = UD_SF_VINA;
    S.weights = {-0.035579f, -0.005156f, 0.840245f, -0.035069f, -0.587439f, 50.0f, 0.05846f};
    S.params.min_rmsd = 0.0f;
    S.params.energy_range = 3.0f;
    S.params.use_graph = 0;  // each batch is searched once
    const Json cfg = read_json(config);
    if (cfg.kind != Json::Object) throw std::runtime_error("paired batch config " + config + " is not a JSON object");
    std::vector<PairedComplex> complexes;
    for (auto& m : cfg.members) {
        const Json *pr = m.second.get("protein"), *lg = m.second.get("ligand"), *lc = m.second.get("ligand_config");
        if (!pr || !lg || !lc) continue;
        PairedComplex c;
        c.protein = pr->str;
        c.ligand = lg->str;
        if (read_ligand_config(lc->str, box, c)) complexes.push_back(c);
        if (complexes.size() >= 5000) {
            std::cout << "Limiting number of ranked samples to max limits 5000\n";
            break;
        }
    }
    std::cout << "Found " << complexes.size() << " to be primed.\n";
    if (complexes.empty()) {
        std::cout << "m_successful_property_count = 0\n";
        return -1;
    }
    const int n_batches = (int)((complexes.size() + batch_size - 1) / batch_size);
    std::cout << "Parameters: exh = " << S.params.exhaustiveness << ", box[0] = " << box[0]
              << ", max_eval_steps global = " << S.params.max_step << ", num_modes = " << S.params.num_modes
              << ", refine_steps = " << S.params.refine_step << "\n";
    std::cout << "To do [" << n_batches << "] batches\n";
    const int n_streams = std::min(batch_size, 16);
    std::vector<cudaStream_t> streams(n_streams);
    for (auto& st : streams)
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
            throw std::runtime_error("could not create a CUDA stream");
    int errors = 0;
    for (int bi = 0; bi < n_batches; ++bi) {
        struct Job {
            const PairedComplex* c = nullptr;
            ud_maps maps = nullptr;
            ud_ligand lig = nullptr;
            ud_batch b = nullptr;
            cudaStream_t s = nullptr;
            bool ok = false;
        };
        std::vector<Job> jobs;
        int batch_errors = 0;
        // complexes of the batch with the same receptor file and box share one set of maps
        std::map<std::string, ud_maps> maps_of;
        for (size_t k = (size_t)bi * batch_size; k < std::min(complexes.size(), (size_t)(bi + 1) * batch_size); ++k) {
            Job j;
            j.c = &complexes[k];
            j.s = streams[jobs.size() % n_streams];
            std::cout << "Processing " << j.c->ligand << "\n";
            try {
                if (!file_exists(j.c->ligand)) throw std::runtime_error("Input ligand file does not exist (" + j.c->ligand + ")");
                if (!file_exists(j.c->protein))
                    throw std::runtime_error("Input (rigid) protein file does not exist (" + j.c->protein + ")");
                Setup Sk = S;
                for (int q = 0; q < 3; ++q) {
                    Sk.center[q] = j.c->center[q];
                    Sk.size[q] = j.c->size[q];
                }
                std::ostringstream key;
                key << j.c->protein << ' ' << Sk.center[0] << ' ' << Sk.center[1] << ' ' << Sk.center[2] << ' '
                    << Sk.size[0] << ' ' << Sk.size[1] << ' ' << Sk.size[2];
                auto it = maps_of.find(key.str());
                if (it == maps_of.end()) it = maps_of.emplace(key.str(), build_maps(Sk, j.c->protein)).first;
                j.maps = it->second;
                auto parsed = parse_ligands({j.c->ligand}, 1, 1);
                if (parsed.empty()) throw std::runtime_error("could not parse " + j.c->ligand);
                j.lig = parsed[0].h;
                check(ud_batch_create(j.maps, &j.lig, 1, j.s, &j.b), "batch");
                check(ud_search_launch(j.b, &S.params, j.s), "search");
                j.ok = true;
            } catch (const std::exception& e) {
                std::cerr << "Exception processing " << j.c->ligand << ", " << e.what() << "\n";
                ++batch_errors;
            }
            jobs.push_back(j);
        }
        for (auto& j : jobs) {
            if (j.ok) {
                try {
                    check(ud_search_collect(j.b, j.s), "search");
                    int n = 0;
                    check(ud_result_count(j.b, 0, &n), "results");
                    if (n == 0) {
                        std::cerr << "WARNING: Could not find any poses. No poses were written.\n";
                    } else {
                        const std::string name = default_output(get_filename(j.c->ligand), dir + "/");
                        write_text(name, result_text(j.b, 0, ends_with(name, ".sdf") ? 1 : 0));
                        float pose[7 + 64], en[8];
                        check(ud_result_mode(j.b, 0, 0, pose, en), "results");
                        std::ostringstream sc;
                        sc << "affinity(kcal/mol)[0]=" << en[0] << "\n";
                        write_text(dir + "/" + default_score_output(get_filename(j.c->ligand)), sc.str());
                    }
                } catch (const std::exception& e) {
                    std::cerr << "Exception processing " << j.c->ligand << ", " << e.what() << "\n";
                    ++batch_errors;
                }
            }
            if (j.b) ud_batch_destroy(j.b);
            if (j.lig) ud_ligand_destroy(j.lig);
        }
        for (auto& m : maps_of) ud_maps_destroy(m.second);
        errors += batch_errors;
        std::cout << "Batch [" << bi + 1 << "/" << n_batches << "] completed. " << batch_errors << " errors.\n";
    }
    for (auto& st : streams) cudaStreamDestroy(st);
    std::cout << errors << " Total errors\n";
    return errors;
}

int run(int argc, char** argv) {
    Options o;
    parse_args(argc, argv, o);
    if (o.has("config")) parse_config(o.str("config"), o);
    if (o.has("help") || o.has("help_advanced") || argc == 1) {
        usage(o.has("help_advanced"));
        return 0;
    }
    if (o.has("version")) {
        std::cout << "unidock (B200 engine, C ABI version " << ud_version() << ")\n";
        return 0;
    }
    for (const char* unsupported : {"flex", "randomize_only"})
        if (o.has(unsupported))
            throw std::runtime_error(std::string("--") + unsupported + " is not supported by this engine");
    Setup S;
    const std::string sf_name = o.str("scoring", "vina");
    if (sf_name == "vina") {
        S.sf = UD_SF_VINA;
        S.weights = {(float)o.num("weight_gauss1", -0.035579), (float)o.num("weight_gauss2", -0.005156),
                     (float)o.num("weight_repulsion", 0.840245), (float)o.num("weight_hydrophobic", -0.035069),
                     (float)o.num("weight_hydrogen", -0.587439), (float)o.num("weight_glue", 50),
                     (float)o.num("weight_rot", 0.05846)};
    } else if (sf_name == "vinardo") {
        S.sf = UD_SF_VINARDO;
        S.weights = {(float)o.num("weight_vinardo_gauss1", -0.045), (float)o.num("weight_vinardo_repulsion", 0.8),
                     (float)o.num("weight_vinardo_hydrophobic", -0.035),
                     (float)o.num("weight_vinardo_hydrogen", -0.6), (float)o.num("weight_glue", 50),
                     (float)o.num("weight_vinardo_rot", o.num("weight_rot", 0.05846))};
    } else if (sf_name == "ad4") {
        S.sf = UD_SF_AD4;
        S.weights = {(float)o.num("weight_ad4_vdw", 0.1662), (float)o.num("weight_ad4_hb", 0.1209),
                     (float)o.num("weight_ad4_elec", 0.1406), (float)o.num("weight_ad4_dsolv", 0.1322),
                     (float)o.num("weight_glue", 50), (float)o.num("weight_ad4_rot", 0.2983)};
    } else {
        throw std::runtime_error("Scoring function " + sf_name + " unknown.");
    }
    const bool score_only = o.has("score_only"), local_only = o.has("local_only");
    S.verbosity = (int)o.num("verbosity", 1);
    const int cpu = (int)o.num("cpu", 0);
    S.threads = cpu > 0 ? cpu : (int)std::max(1u, std::thread::hardware_concurrency());
    S.spacing = (float)o.num("spacing", 0.375);
    S.autotune = o.has("autotune");
    S.multi_bias = o.has("multi_bias");
    if (S.multi_bias && S.sf == UD_SF_AD4)
        throw std::runtime_error("--multi_bias with --scoring ad4 is not supported by this engine");
    // search parameters and search_mode presets (main.cpp:644-661)
    const bool batch_mode = o.has("gpu_batch") || o.has("batch") || o.has("ligand_index");
    int exhaustiveness = (int)o.num("exhaustiveness", 8);
    int max_step = (int)o.num("max_step", 0);
    if (o.has("search_mode")) {
        const std::string m = o.str("search_mode");
        if (m == "balance" || m == "balanced") {
            exhaustiveness = 384;
            max_step = 40;
        } else if (m == "fast") {
            exhaustiveness = 128;
            max_step = 20;
        } else if (m == "detail" || m == "detailed") {
            exhaustiveness = 512;
            max_step = 40;
        } else {
            throw std::runtime_error("unknown search_mode " + m + " (fast, balance, detail)");
        }
    } else if (batch_mode && !o.has("exhaustiveness")) {
        exhaustiveness = 384;
        max_step = 40;
    }
    if (exhaustiveness < 1) throw std::runtime_error("exhaustiveness must be 1 or greater");
    ud_search_params& p = S.params;
    p.exhaustiveness = exhaustiveness;
    p.max_step = max_step;
    p.num_modes = (int)o.num("num_modes", 9);
    p.min_rmsd = (float)o.num("min_rmsd", 1.0);
    p.energy_range = (float)o.num("energy_range", 3.0);
    p.seed = (unsigned long long)(long long)o.num("seed", 0);
    p.form = 1;
    p.chains_per_block = 0;
    p.bfgs_cap = 0;
    p.use_graph = 1;
    const bool no_refine = o.has("no_refine");
    p.refine_step = no_refine ? 0 : (int)o.num("refine_step", 3);
    // one-ligand-one-protein batches (main.cpp:663-700)
    const int paired_batch_size = (int)o.num("paired_batch_size", 0);
    if (paired_batch_size > 0) {
        if (!o.has("ligand_index")) {
            std::cout << "ERROR: Paired batch size set, but no config json specified via --ligand_index\n";
            return -1;
        }
        float box[3] = {25, 25, 25};
        if (!o.has("size_x") || !o.has("size_y") || !o.has("size_z"))
            std::cout << "WARN: Paired batch size set, but size_x/size_y/size_z not specified, using 25\n";
        else
            box[0] = (float)o.num("size_x", 25), box[1] = (float)o.num("size_y", 25), box[2] = (float)o.num("size_z", 25);
        if (!o.has("dir")) {
            std::cout << "ERROR: Need to specify an output directory for batch mode.\n";
            return -1;
        }
        std::cout << "Entering paired batch mode\n";
        const int device = (int)o.num("device_id", 0);
        if (cudaSetDevice(device) != cudaSuccess) throw std::runtime_error("could not select GPU " + std::to_string(device));
        return run_paired(S, o.str("ligand_index"), o.str("dir"), paired_batch_size, box, local_only);
    }
    if (!o.has("receptor") && !o.has("maps")) throw std::runtime_error("The receptor or affinity maps must be specified.");
    // ligands
    std::vector<std::string> ligand_names = o.list("ligand");
    std::vector<std::string> batch_names = o.list("gpu_batch");
    for (auto& n : o.list("batch")) batch_names.push_back(n);
    if (o.has("ligand_index")) {
        std::ifstream idx(o.str("ligand_index"));
        if (!idx) throw std::runtime_error("could not open \"" + o.str("ligand_index") + "\" for reading");
        for (std::string n; idx >> n;) batch_names.push_back(n);
    }
    if (ligand_names.empty() && batch_names.empty()) throw std::runtime_error("Missing ligand(s).");
    if (!ligand_names.empty() && (o.has("batch") || o.has("gpu_batch")))
        throw std::runtime_error("Can't use both --ligand and --batch arguments simultaneously.");
    const std::string dir = o.str("dir");
    if (batch_mode && !o.has("dir")) throw std::runtime_error("Need to specify an output directory for batch mode.");
    if (o.has("dir") && !is_directory(dir)) throw std::runtime_error("Directory " + dir + " does not exist.");
    if (ligand_names.size() > 1) throw std::runtime_error("docking several --ligand files together is not supported "
                                                          "by this engine; use --gpu_batch");
    // box
    const bool autobox = o.has("autobox");
    for (int i = 0; i < 3; ++i) {
        const char* c[3] = {"center_x", "center_y", "center_z"};
        const char* z[3] = {"size_x", "size_y", "size_z"};
        if (!autobox && !o.has("maps") && (!o.has(c[i]) || !o.has(z[i])))
            throw std::runtime_error("the search space (--center_x/y/z, --size_x/y/z) must be specified");
        S.center[i] = (float)o.num(c[i], 0);
        S.size[i] = (float)o.num(z[i], 0);
    }
    if (autobox) {
        if (!(score_only || local_only) || ligand_names.empty())
            throw std::runtime_error("--autobox is for --score_only and --local_only with --ligand");
        // Vina::grid_dimensions_from_ligand with a 4 A buffer (main.cpp:368, vina.cpp:460-488)
        std::string t = read_file(ligand_names[0]);
        ud_ligand h = nullptr;
        check(ud_ligand_parse(t.data(), t.size(), &h), "ligand");
        int counts[8];
        check(ud_ligand_counts(h, counts), "ligand");
        std::vector<float> lab(3 * (size_t)counts[0]);
        check(ud_ligand_export(h, lab.data(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                               nullptr, nullptr, nullptr, nullptr),
              "ligand");
        ud_ligand_destroy(h);
        for (int i = 0; i < 3; ++i) {
            double c = 0, m = 0;
            for (int a = 0; a < counts[0]; ++a) c += lab[3 * a + i];
            c /= std::max(1, counts[0]);
            for (int a = 0; a < counts[0]; ++a) m = std::max(m, std::fabs(c - lab[3 * a + i]));
            S.center[i] = (float)c;
            S.size[i] = (float)std::ceil((m + 4.0) * 2);
        }
    }
    for (int i = 0; i < 3 && !o.has("maps"); ++i) {
        if (!(S.size[i] > 0)) throw std::runtime_error("Grid box dimensions must be greater than 0 Angstrom.");
        if (o.has("force_even_voxels")) {  // vina.cpp:529-534: odd voxel counts get one more voxel
            long nv = (long)std::ceil(S.size[i] / S.spacing);
            if (nv % 2 == 1) S.size[i] = (float)((nv + 1) * (double)S.spacing);
        }
    }
    if ((double)S.size[0] * S.size[1] * S.size[2] > 27e3)
        std::cerr << "WARNING: Search space volume is greater than 27000 Angstrom^3 (See FAQ)\n";
    if (S.verbosity > 0) {
        std::cout << "Scoring function : " << sf_name << "\n";
        if (o.has("receptor")) std::cout << "Rigid receptor: " << o.str("receptor") << "\n";
        if (o.has("maps")) std::cout << "Affinity maps: " << o.str("maps") << "\n";
        if (ligand_names.size() == 1) std::cout << "Ligand: " << ligand_names[0] << "\n";
        else std::cout << "Ligands (batch mode): " << batch_names.size() << " molecules\n";
        std::cout << std::setprecision(6) << "Grid center: X " << S.center[0] << " Y " << S.center[1] << " Z "
                  << S.center[2] << "\n";
        std::cout << "Grid size  : X " << S.size[0] << " Y " << S.size[1] << " Z " << S.size[2] << "\n";
        std::cout << "Grid space : " << S.spacing << "\n";
        std::cout << "Exhaustiveness: " << exhaustiveness << "\n";
        std::cout << "CPU: " << cpu << "\n";
        std::cout << "Seed: " << p.seed << "\n";
        std::cout << "Verbosity: " << S.verbosity << "\n\n";
    }
    const int device = (int)o.num("device_id", 0);
    if (cudaSetDevice(device) != cudaSuccess) throw std::runtime_error("could not select GPU " + std::to_string(device));
    size_t free_start = 0, total_mem = 0;
    cudaFree(nullptr);  // the context, so that its own memory is not counted below
    cudaMemGetInfo(&free_start, &total_mem);
    ud_maps maps = nullptr;
    if (o.has("maps")) {
        check(ud_maps_load(S.sf, S.weights.data(), (int)S.weights.size(), o.str("maps").c_str(), nullptr, &maps),
              "maps");
        if (o.has("bias") && S.sf == UD_SF_AD4) {  // AD4.2 maps read, then ad4cache::set_bias (vina.cpp:577-586)
            const std::string bpf = read_file(o.str("bias"));
            check(ud_maps_add_bias(maps, bpf.data(), bpf.size(), nullptr), "bias");
        }
    } else {
        maps = build_maps(S, o.str("receptor"));
        S.receptor_scoring = !no_refine && S.sf != UD_SF_AD4;
        if (o.has("bias")) {  // Vina::set_bias, then the wells go into the maps (vina.cpp:547-553)
            const std::string bpf = read_file(o.str("bias"));
            check(ud_maps_add_bias(maps, bpf.data(), bpf.size(), nullptr), "bias");
        }
    }
    if (o.has("write_maps")) check(ud_maps_write(maps, o.str("write_maps").c_str()), "write maps");
    if (!ligand_names.empty()) {
        std::string out_name = o.has("out") ? o.str("out") : default_output(ligand_names[0]);
        if (!score_only && S.verbosity > 0 && !o.has("out")) std::cout << "Output will be " << out_name << "\n";
        run_single(S, maps, ligand_names[0], out_name, score_only, local_only);
    } else if (score_only || local_only) {
        // batch scoring / local optimisation: one ligand at a time, as the reference's batch --score_only
        std::ofstream sfile;
        if (score_only) sfile.open(dir + "/" + o.str("score_file", "scores.txt"));
        auto ligs = parse_ligands(batch_names, S.threads, S.verbosity);
        for (auto& L : ligs) {
            ud_batch b = nullptr;
            check(ud_batch_create(maps, &L.h, 1, nullptr, &b), "batch");
            int counts[8];
            check(ud_ligand_counts(L.h, counts), "ligand");
            std::vector<float> pose(7 + counts[2]);
            check(ud_ligand_initial_pose(L.h, pose.data()), "ligand");
            float en[8];
            if (local_only) local_optimize(maps, b, L.h, pose);
            score_pose(S, b, pose, en);
            if (score_only)
                sfile << get_filename(L.path) << " " << std::fixed << std::setprecision(3) << en[0] << "\n";
            if (S.verbosity > 0) print_energies(std::cout, en);
            ud_batch_destroy(b);
            ud_ligand_destroy(L.h);
        }
    } else {
        const int batch_size = std::max(1, (int)o.num("batch_size", 4096));
        // --max_gpu_memory (MiB; 0 = 95% of the free memory, main.cpp:955-965):
        // what the maps left, less a reserve for the receptor cells and the
        // search set-up, is shared by the two batches in flight
        size_t free_now = 0;
        cudaMemGetInfo(&free_now, &total_mem);
        const size_t used = free_start > free_now ? free_start - free_now : 0;
        const double max_mib = o.num("max_gpu_memory", 0);
        const size_t reserve = (size_t)64 << 20;
        size_t slot_budget = 0;
        if (max_mib > 0) {
            const size_t cap = (size_t)(max_mib * 1048576.0);
            if (cap <= used + reserve)
                throw std::runtime_error("--max_gpu_memory " + std::to_string((long long)max_mib) +
                                         " MiB is below the maps' own " + std::to_string(used >> 20) + " MiB");
            slot_budget = (cap - used - reserve) / 2;
        } else {
            slot_budget = (size_t)(0.95 * (double)free_now) / 2;
        }
        if (S.verbosity > 1)
            std::cout << "GPU memory: maps " << (used >> 20) << " MiB, per batch " << (slot_budget >> 20) << " MiB\n";
        run_batches(S, maps, batch_names, dir, batch_size, slot_budget);
    }
    ud_maps_destroy(maps);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {
        std::cerr << "\n\nERROR: " << e.what() << "\n";
        return 1;
    }
}
