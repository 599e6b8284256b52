// fluidsim_home: drop-in for the reference's headless fluidsim_home
// (src/apps/main_home.cpp), same flags and outputs, on liblbm_b200.
#include "sim_host.hpp"

int main(int argc, char** argv) { return fsim::cli_main(argc, argv, LBM_METHOD_HOME, "home"); }
