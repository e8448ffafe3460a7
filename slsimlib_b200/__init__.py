"""B200-native GLAMER ray-shooting path."""
