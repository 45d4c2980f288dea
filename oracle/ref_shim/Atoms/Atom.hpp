// Build shim (test infrastructure only): the reference's Atoms/Atom.hpp
// declares PETSc-bound set-up functions that the shim-compiled arithmetic
// files never call; only Macros.hpp is needed from it.
#ifndef BTAM_REF_SHIM_ATOM_HPP
#define BTAM_REF_SHIM_ATOM_HPP
#include "Macros.hpp"
#include <vector>
using namespace std;
#endif
