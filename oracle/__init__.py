"""CPU oracle (test infrastructure): C restatement + the reference compiled from source."""
