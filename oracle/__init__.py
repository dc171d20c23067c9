"""CPU checkers (test infrastructure): the oracle restatement and the reference harness."""
