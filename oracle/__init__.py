"""CPU oracle for the ursa-core hot path (test infrastructure; see oracle.py)."""
