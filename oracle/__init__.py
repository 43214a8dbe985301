"""CPU oracle of the OERM Monte Carlo path (test infrastructure only)."""
