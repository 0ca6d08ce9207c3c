"""cm1_b200: B200-native dynamical-core large step of CM1 (see include/cm1g.h)."""
