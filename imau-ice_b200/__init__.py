"""B200-native ice-velocity hot path of IMAU-ICE (DIVA / SSA / SIA).

Modules:
  diva   -- reference-shaped host API (Grid, Context, solve_SIA/SSA/DIVA)
  synth  -- seeded synthetic geometries of the benchmark configurations
  build  -- nvcc build of lib/libdiva_b200.so (sm_100a)
"""
