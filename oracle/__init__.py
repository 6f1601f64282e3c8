"""CPU oracle of the livox-warp hot path (test infrastructure only; see oracle.py)."""
