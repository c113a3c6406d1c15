// Builds the reference's ColocSim::assemble_matrices (Bem/Simulation/ColocSim.cpp) from its
// unmodified source with the wall image switched off.  The reference selects the image
// kernel with `#define MIRROR_MESH true` (Bem/Simulation/LinLinSim.hpp:13); including the
// header first and redefining the macro before the .cpp is compiled keeps the source as it is.
#include "Bem/Simulation/LinLinSim.hpp"
#undef MIRROR_MESH
#define MIRROR_MESH false
#include "Bem/Simulation/ColocSim.cpp"
