"""grasph2_b200: GraSPH2's per-step hot path on the NVIDIA B200 (sm_100a)."""
