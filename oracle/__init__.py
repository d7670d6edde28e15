"""CPU oracle (test infrastructure): C restatement of the reference hot path."""
