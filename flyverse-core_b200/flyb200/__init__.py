"""flyb200: B200-native per-step brain update (event-driven LIF + optic lobe)."""
