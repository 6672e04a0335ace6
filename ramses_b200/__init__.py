"""B200-native RAMSES hydro step (unsplit MUSCL-Hancock on the AMR octree)."""
