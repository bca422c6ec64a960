"""croma-fp_b200: B200-native tracer Fokker-Planck update (drop-in for the
CUDA backend of kosukenishiwaki/croma-fp)."""
