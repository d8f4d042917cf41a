"""B200-native (sm_100a) implementation of FINFLO's per-iteration hot path."""
