"""CPU oracle for the dedisp hot path -- test infrastructure only (see oracle.h)."""
