"""cunibs_b200: B200-native per-placement TMS field solve, a drop-in for cuNIBS's forward path."""
