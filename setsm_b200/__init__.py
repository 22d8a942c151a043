"""B200-native SETSM vertical-line-locus matcher (see include/setsm_vll.h)."""
