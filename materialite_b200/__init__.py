"""materialite_b200: sm_100a SmallStrainFFT solve with materialite's plugin API."""
