"""CPU oracle of the detector (test infrastructure only; see rtod_oracle.cpp)."""
