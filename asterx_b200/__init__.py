"""asterx_b200: B200-native GRMHD right-hand-side and primitive-recovery
engine (host-side Python helpers; the engine itself is the C ABI in
``include/asterx_b200.h``, built into ``asterx_b200/_lib``)."""
