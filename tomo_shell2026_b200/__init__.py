"""B200-native orientation search (rotate -> voxelize -> slot-pair -> shadow-cast -> reduce -> argmin)."""
