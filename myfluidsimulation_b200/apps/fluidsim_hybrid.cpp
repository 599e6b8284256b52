// fluidsim_hybrid: drop-in for the reference's headless fluidsim_hybrid
// (src/apps/main_hybrid.cpp), same flags and outputs, on liblbm_b200.
#include "sim_host.hpp"

int main(int argc, char** argv) { return fsim::cli_main(argc, argv, LBM_METHOD_HYBRID, "hybrid"); }
