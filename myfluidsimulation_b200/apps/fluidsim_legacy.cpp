// fluidsim_legacy: drop-in for the reference's headless fluidsim_legacy
// (src/apps/main_legacy.cpp), same flags and outputs, on liblbm_b200.
#include "sim_host.hpp"

int main(int argc, char** argv) { return fsim::cli_main(argc, argv, LBM_METHOD_LEGACY, "legacy"); }
