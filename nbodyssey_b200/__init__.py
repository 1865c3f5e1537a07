"""nbodyssey_b200: B200-native force-and-step path of nbodyssey."""
