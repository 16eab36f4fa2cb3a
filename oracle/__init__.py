"""CPU oracle of the voxel-hashing TSDF pipeline - test infrastructure only."""
