// Build shim (test infrastructure only): empty stand-in for petscerror.h.
