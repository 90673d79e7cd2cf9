"""B200-native EAM force-and-stress path for mdelast (see DESIGN.md for the layout)."""
