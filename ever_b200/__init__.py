"""B200-native exact volumetric ellipsoid tracer (drop-in for EVER's trace_rays)."""
