"""B200-native liquid step (drop-in for the reference LiquidModel<3>/CGSolver<3>)."""
