"""Placeholder colormap module."""
viridis = None
