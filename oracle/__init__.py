"""CPU oracle and reference bindings -- test infrastructure only (see awp_oracle.h)."""
