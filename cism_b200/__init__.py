"""B200-native Blatter-Pattyn velocity solver (CISM glissade_velo_higher)."""
