"""CPU oracle (test infrastructure only; see lym_oracle.py)."""
