// Handles shared by the test-only reference drivers (ref_driver.cpp over the
// reference's CPU sources, ref_gpu_driver.cu over its CUDA search): receptor
// maps and parsed ligands built by the reference's own code.
#pragma once
#include <memory>

#include "ad4cache.h"
#include "bias.h"
#include "cache.h"
#include "model.h"
#include "non_cache.h"
#include "precalculate.h"
#include "scoring_function.h"

struct RefMaps {
    std::shared_ptr<ScoringFunction> sf;
    std::unique_ptr<precalculate> pre;
    model rec;
    cache grid;
    ad4cache ad4;               // AutoDock 4.2 maps read from .map files
    const igrid* ig = &grid;    // the maps the model is scored against
    grid_dims gd;
    std::unique_ptr<non_cache> nc;  // explicit receptor atoms, built on first use
    std::vector<bias_element> bias; // wells added to the maps and to non_cache
    vec corner1() const { return ig == &grid ? grid.corner1() : ad4.corner1(); }
    vec corner2() const { return ig == &grid ? grid.corner2() : ad4.corner2(); }
};

struct RefLigand {
    std::shared_ptr<ScoringFunction> sf;
    model m;
    std::unique_ptr<precalculate_byatom> pre;
    std::vector<bias_element> bias; // the ligand's own wells (model::bias_list of its docking model)
};

