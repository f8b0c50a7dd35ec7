// udref_dock.cpp -- runs the reference docking engine (Uni-Dock2's core_pipeline, compiled
// from the reference sources by oracle/Makefile into oracle/_ref/udref_dock) on one input
// file of the reference's JSON schema, with the parameters the Python DockingPipeline
// passes (api/python/pipeline.cpp:58-144).  Test infrastructure: it times the reference's
// own CUDA engine on the same GPU as this engine; nothing of the product calls it.
//
//   udref_dock input.json out_dir cx cy cz sx sy sz exhaustiveness mc_steps opt_steps
//              refine_steps num_pose rmsd_limit energy_range seed constraint
//              [energy_decomp [bias bias_k]]      (bias: no | pos | align)
//
// Prints one JSON line: {"rc", "ligands", "seconds"} (wall time of core_pipeline).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>

#include "format/json.h"
#include "screening/core.h"

int main(int argc, char** argv) {
    if (argc != 18 && argc != 19 && argc != 21) {
        std::fprintf(stderr, "usage: udref_dock input.json out_dir cx cy cz sx sy sz exhaustiveness mc_steps "
                             "opt_steps refine_steps num_pose rmsd_limit energy_range seed constraint "
                             "[energy_decomp [bias bias_k]]\n");
        return 2;
    }
    std::ifstream f(argv[1]);
    std::stringstream ss;
    ss << f.rdbuf();
    CoreInput ipt;
    ipt.output_dir = argv[2];
    ipt.name_json = "udref";
    const float cx = std::atof(argv[3]), cy = std::atof(argv[4]), cz = std::atof(argv[5]);
    const float sx = std::atof(argv[6]), sy = std::atof(argv[7]), sz = std::atof(argv[8]);
    ipt.box.x_lo = cx - sx / 2; ipt.box.x_hi = cx + sx / 2;
    ipt.box.y_lo = cy - sy / 2; ipt.box.y_hi = cy + sy / 2;
    ipt.box.z_lo = cz - sz / 2; ipt.box.z_hi = cz + sz / 2;
    ipt.task = "screen";
    ipt.search_mode = "free";
    ipt.exhaustiveness = std::atoi(argv[9]);
    ipt.mc_steps = std::atoi(argv[10]);
    ipt.opt_steps = std::atoi(argv[11]);
    ipt.refine_steps = std::atoi(argv[12]);
    ipt.num_pose = std::atoi(argv[13]);
    ipt.rmsd_limit = std::atof(argv[14]);
    ipt.energy_range = std::atof(argv[15]);
    ipt.seed = std::atoi(argv[16]);
    ipt.constraint_docking = std::atoi(argv[17]) != 0;
    ipt.energy_decomp = argc >= 19 && std::atoi(argv[18]) != 0;
    if (argc == 21) {
        ipt.bias = argv[19];
        ipt.bias_k = std::atof(argv[20]);
    }
    ipt.randomize = true;
    read_ud_from_json_string(ss.str(), ipt.box, ipt.fix_mol, ipt.flex_mol_list, ipt.fns_flex, false);
    const size_t nlig = ipt.flex_mol_list.size();
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = core_pipeline(ipt);
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("{\"rc\": %d, \"ligands\": %zu, \"seconds\": %.3f}\n", rc, nlig, sec);
    return rc;
}
