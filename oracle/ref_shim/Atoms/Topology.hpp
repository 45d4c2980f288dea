// Build shim (test infrastructure only): stands in for the reference's
// Atoms/Topology.hpp, whose PETSc IS-based declarations are not needed here.
#ifndef BTAM_REF_SHIM_TOPOLOGY_HPP
#define BTAM_REF_SHIM_TOPOLOGY_HPP
#include "Macros.hpp"
#endif
