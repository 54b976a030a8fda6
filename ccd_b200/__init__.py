"""ccd_b200: B200-native cyclic coordinate descent for Cyclops-style regressions."""
