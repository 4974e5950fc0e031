"""CPU oracles of the fermion hot path -- TEST INFRASTRUCTURE (tests, smoke and the CPU baseline only)."""
