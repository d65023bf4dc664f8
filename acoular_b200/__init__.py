"""B200-native frequency-domain beamforming for Acoular (CSM estimation + steered-response map)."""
