// heat_solver_b200 -- drop-in command line for the reference solver binary
// (src/heat_solver_het.cu main, het.cu:1355-1629); all work is in libheat_b200.
#include "../../include/heat_b200.h"

int main(int argc, char** argv) { return hs_cli_main(argc, argv); }
