"""Mesh generation (synthetic channels) and device mesh handles."""
