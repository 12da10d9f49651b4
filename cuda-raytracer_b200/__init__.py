"""B200-native Radiance path tracer (drop-in for xlnx/cuda-raytracer's Radiance path)."""
