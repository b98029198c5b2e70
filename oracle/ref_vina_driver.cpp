// Test-only C interface over the REFERENCE's stock CPU docking path, compiled
// from its own sources by oracle/Makefile into oracle/_ref/libudref_gpu.so
// (vina.cpp and parallel_mc.cpp need the host code of its monte_carlo.cu):
//   udref_vina_dock    the whole CPU docking of one ligand, as the reference
//                      CLI runs it with --cpu: Vina::set_receptor,
//                      set_ligand_from_file, compute_vina_maps,
//                      global_search (vina.cpp:1495-1653: parallel_mc over
//                      the heuristic step count, refinement, rescoring);
//   udref_parallel_mc  the same parallel Monte-Carlo machinery (parallel_mc
//                      over monte_carlo::operator(), parallel_mc.cpp:68-79,
//                      monte_carlo.cu:2319-2356) with the step count set to a
//                      cap, as the reference's GPU path applies --max_step.
// Only tests and the CPU legs of bench.py load this.
#include <cstring>

#include "parallel_mc.h"
#include "ref_driver.h"
#include "vina.h"

extern "C" {

int udref_vina_dock(const char* receptor, const char* ligand, const float* center, const float* size, float spacing,
                    int exhaustiveness, int n_poses, int seed, int threads, double* out_e, int n_out) {
    try {
        Vina v("vina", threads, seed, 0);
        v.set_receptor(receptor);
        v.set_ligand_from_file(std::string(ligand));
        v.compute_vina_maps(center[0], center[1], center[2], size[0], size[1], size[2], spacing);
        v.global_search(exhaustiveness, n_poses, 1.0, 0);
        const std::vector<std::vector<double> > e = v.get_poses_energies(n_poses, 3.0);
        const int n = std::min<int>((int)e.size(), n_out);
        for (int i = 0; i < n; ++i) out_e[i] = e[i].empty() ? 0.0 : e[i][0];
        return n;
    } catch (...) {
        return -1;
    }
}

int udref_parallel_mc(void* lh, void* mh, int exhaustiveness, int global_steps, unsigned seed, int threads,
                      int n_saved, float min_rmsd, float* out_e, float* out_pose, int pose_stride) {
    try {
        auto L = (RefLigand*)lh;
        auto M = (RefMaps*)mh;
        parallel_mc pmc;
        pmc.mc.global_steps = (unsigned)global_steps;
        pmc.mc.local_steps = unsigned((25 + L->m.num_movable_atoms()) / 3);
        pmc.mc.max_evals = 0;
        pmc.mc.min_rmsd = min_rmsd;
        pmc.mc.num_saved_mins = (sz)n_saved;
        pmc.mc.hunt_cap = vec(10, 10, 10);
        pmc.num_tasks = (sz)exhaustiveness;
        pmc.num_threads = (sz)threads;
        pmc.display_progress = false;
        output_container out;
        rng generator(static_cast<rng::result_type>(seed));
        pmc(L->m, out, *L->pre, *M->ig, M->corner1(), M->corner2(), generator);
        const int n = std::min<int>((int)out.size(), n_saved);
        for (int i = 0; i < n; ++i) {
            out_e[i] = out[i].e;
            if (out_pose) {
                const auto& r = out[i].c.ligands[0].rigid;
                float* p = out_pose + (size_t)i * pose_stride;
                for (int k = 0; k < 3; ++k) p[k] = r.position[k];
                p[3] = r.orientation.R_component_1();
                p[4] = r.orientation.R_component_2();
                p[5] = r.orientation.R_component_3();
                p[6] = r.orientation.R_component_4();
                const auto& t = out[i].c.ligands[0].torsions;
                for (size_t k = 0; k < t.size(); ++k) p[7 + k] = t[k];
            }
        }
        return n;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
