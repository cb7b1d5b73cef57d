"""Drop-in counterparts of AstroFD's utils/ modules on the device path."""
