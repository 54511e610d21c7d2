"""CPU FP64 oracle of the reference's Biot-Savart / RK4 path (test infrastructure only)."""
