"""MaBoSS-compatible stochastic Boolean network simulation."""
