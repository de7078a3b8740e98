"""CPU parity oracle (test infrastructure only; see oracle.cpp)."""
