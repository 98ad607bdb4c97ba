"""Bunch and profile monitors (blond/monitors) with device-side buffers."""
