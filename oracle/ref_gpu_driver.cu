// Test-only C interface over the REFERENCE's own GPU batched search
// (unidock/src/cuda/monte_carlo.cu: monte_carlo_template::do_docking<Config>,
// unidock/src/cuda/precalculate.cu: precalculate_parallel), compiled for
// sm_100a by oracle/Makefile into oracle/_ref/libudref_gpu.so.  It times the
// reference's kernel on the same GPU as the engine; nothing in the product
// links it.
//
// Set-up follows Vina::set_ligand_from_object_gpu (unidock/src/lib/vina.cpp:
// 246-303) and the search parameters of Vina::global_search_gpu
// (unidock/src/lib/vina.h:154-230); the size bucket (Config) is chosen per
// call, as unidock/src/main/main.cpp:95-118 groups ligands, but from the
// limits the kernel's fixed-size arrays actually have (unidock/src/cuda/
// kernel.h: atoms, torsions, rigid bodies, intramolecular pairs), so that no
// ligand can overflow them.
#include <chrono>
#include <cmath>
#include <string>
#include <vector>

#include "kernel.h"
#include "monte_carlo.h"
#include "ref_driver.h"

namespace {
thread_local std::string g_gpu_err;

struct Limits {
    size_t atoms, torsions, rigids, pairs;
};
template <class C> Limits limits_of() {
    return Limits{C::MAX_NUM_OF_ATOMS_, C::MAX_NUM_OF_LIG_TORSION_, C::MAX_NUM_OF_RIGID_, C::MAX_NUM_OF_LIG_PAIRS_};
}

bool fits(const model& m, const Limits& L) {
    const ligand& lig = m.ligands[0];
    const size_t torsions = m.get_size().ligands[0];
    return m.num_atoms() < L.atoms && m.num_atoms() < MAX_NUM_OF_ATOMS && torsions <= L.torsions &&
           torsions + 1 <= L.rigids && lig.pairs.size() <= L.pairs;
}
}  // namespace

extern "C" {

const char* udref_gpu_last_error() { return g_gpu_err.c_str(); }

// Smallest size bucket (0 Small, 1 Medium, 2 Large, 3 ExtraLarge, 4 Max) whose
// arrays hold every ligand of the list, or -1.
int udref_gpu_config(void** ligands, int n) {
    const Limits all[5] = {limits_of<SmallConfig>(), limits_of<MediumConfig>(), limits_of<LargeConfig>(),
                           limits_of<ExtraLargeConfig>(), limits_of<MaxConfig>()};
    for (int c = 0; c < 5; ++c) {
        bool ok = true;
        for (int i = 0; i < n && ok; ++i) ok = fits(((RefLigand*)ligands[i])->m, all[c]);
        if (ok) return c;
    }
    return -1;
}

// The reference's GPU search of n ligands against the maps: per-ligand pair
// tables on the device (precalculate_parallel), then do_docking<Config> with
// exhaustiveness chains per ligand.  best_e[i] = energy of ligand i's best
// output pose (NaN when none); t_out[0] = seconds of the pair tables,
// t_out[1] = seconds of do_docking (host marshalling, kernel, copy-back and
// conversion of the results).  Returns the Config used, or -1.
int udref_gpu_dock(void* mh, void** ligands, int n, int exhaustiveness, int max_step, unsigned long long seed,
                   float* best_e, double* t_out) {
    try {
        auto M = (RefMaps*)mh;
        if (n < 1 || n > MAX_LIGAND_NUM || M->ig != &M->grid) {
            g_gpu_err = "invalid arguments";
            return -1;
        }
        const int config = udref_gpu_config(ligands, n);
        if (config < 0) {
            g_gpu_err = "a ligand exceeds every size bucket";
            return -1;
        }
        if ((long long)exhaustiveness * n > MAX_THREAD) {
            g_gpu_err = "too many chains";
            return -1;
        }
        std::vector<model> models(n, M->rec);
        std::vector<precalculate_byatom> pre(n);
        for (int i = 0; i < n; ++i) {
            models[i].append(((RefLigand*)ligands[i])->m);
            pre[i].init_without_calculation(*M->sf, models[i]);
        }
        static triangular_matrix_cuda_t data_list[MAX_LIGAND_NUM];
        flv common_rs = pre[0].calculate_rs();
        auto t0 = std::chrono::steady_clock::now();
        precalculate_parallel(data_list, pre, *M->sf, models, common_rs, n);
        checkCUDA(cudaDeviceSynchronize());
        auto t1 = std::chrono::steady_clock::now();

        monte_carlo_template mc;
        sz heuristic = 0;
        for (int i = 0; i < n; ++i) {
            heuristic = std::max(heuristic, models[i].num_movable_atoms() +
                                                10 * models[i].get_size().num_degrees_of_freedom());
            mc.local_steps = unsigned((25 + models[i].num_movable_atoms()) / 3);
        }
        mc.global_steps = unsigned(70 * 3 * (50 + heuristic) / 2);
        if (max_step > 0 && mc.global_steps > (unsigned)max_step) mc.global_steps = (unsigned)max_step;
        mc.max_evals = 0;
        mc.min_rmsd = 1.0;
        mc.num_saved_mins = 9;
        mc.hunt_cap = vec(10, 10, 10);
        mc.threads_per_ligand = exhaustiveness;
        mc.num_of_ligands = n;
        mc.thread = exhaustiveness * n;
        mc.local_only = false;
        std::vector<output_container> out(n);
        rng generator(static_cast<rng::result_type>(seed));
        std::vector<std::vector<bias_element>> bias;
        const vec c1 = M->grid.corner1(), c2 = M->grid.corner2();
        switch (config) {
            case 0: mc.do_docking<SmallConfig>(models, out, pre, data_list, M->grid, c1, c2, generator, 0, seed, bias); break;
            case 1: mc.do_docking<MediumConfig>(models, out, pre, data_list, M->grid, c1, c2, generator, 0, seed, bias); break;
            case 2: mc.do_docking<LargeConfig>(models, out, pre, data_list, M->grid, c1, c2, generator, 0, seed, bias); break;
            case 3: mc.do_docking<ExtraLargeConfig>(models, out, pre, data_list, M->grid, c1, c2, generator, 0, seed, bias); break;
            default: mc.do_docking<MaxConfig>(models, out, pre, data_list, M->grid, c1, c2, generator, 0, seed, bias); break;
        }
        checkCUDA(cudaDeviceSynchronize());
        auto t2 = std::chrono::steady_clock::now();
        for (int i = 0; i < n; ++i) best_e[i] = out[i].empty() ? NAN : (float)out[i][0].e;
        t_out[0] = std::chrono::duration<double>(t1 - t0).count();
        t_out[1] = std::chrono::duration<double>(t2 - t1).count();
        return config;
    } catch (const std::exception& e) {
        g_gpu_err = e.what();
        return -1;
    }
}

}  // extern "C"
