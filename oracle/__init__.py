"""CPU oracle (test infrastructure only): see ovs_oracle.h."""
