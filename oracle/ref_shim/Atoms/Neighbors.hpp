// Build shim (test infrastructure only): stands in for the reference's
// Atoms/Neighbors.hpp, whose PETSc-bound declarations are not needed here.
#ifndef BTAM_REF_SHIM_NEIGHBORS_HPP
#define BTAM_REF_SHIM_NEIGHBORS_HPP
#include "Macros.hpp"
#endif
