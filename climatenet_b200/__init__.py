"""B200-native projective-dynamics frictional-contact step loop (package root)."""
