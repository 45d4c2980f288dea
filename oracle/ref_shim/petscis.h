// Build shim (test infrastructure only): empty stand-in for petscis.h.
