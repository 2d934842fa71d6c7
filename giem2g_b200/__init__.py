"""B200-native IE-solve hot path of GIEM2G (placeholder, filled in below)."""
