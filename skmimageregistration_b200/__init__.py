"""B200-native evaluation path of Sparse Kernel Machine image registration."""
