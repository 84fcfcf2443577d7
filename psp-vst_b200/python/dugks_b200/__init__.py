"""dugks_b200: B200-native DUGKS step (dugksFoam fvDVM::evolution) behind a C ABI."""
