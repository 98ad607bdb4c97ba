"""RF beam-phase loop (blond/llrf): BeamFeedback with the beam phase on the device."""
