"""B200-native sparse-voxel-tree ray march of the voxel engine
Vuk03-boop/voxelcraft-menu.

Layout:
  csrc/            CUDA kernels (sm_100a), the C ABI and the host world store
  native.py        ctypes binding of libvoxmarch.so
  world.py         World (encoder + pools), cameras, synthetic worlds, views
  march.py         Marcher (one device context) and Renderer (engine interface)
  shading.py       differentiable shading stage (forward / adjoint kernels)
  build.py         builds libvoxmarch.so in-tree
"""
from .world import (AIR, DIRT, FLAG_HEATMAP, FLAG_HIZ, FLAG_SHADOWS, FLAG_UNDERWATER, FLAG_WATER_REFRACT, GLASS,
                    GLOWSTONE, GRASS, LEAVES, LOG, NO_CHUNK, STONE, WATER, Camera, Recipe, View, World,
                    camera_basis, default_sun, dense_index, halton_jitter, large_terrain_camera, pairs_for,
                    recipe_large_terrain, recipe_small_terrain, recipe_sparse_world, small_terrain_camera,
                    surface_height)
from .march import MarchError, Marcher, PairDemand, Renderer

__all__ = [n for n in dir() if not n.startswith("_")]
