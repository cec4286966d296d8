"""Module-level settings the drop-in step reads.

``updates.SRK2_force_calc`` reads the same module globals the reference's
step reads from its ``config`` module (config.py:13-26): the dimension, the
box side, the SRK order, the dt rule's ``max_dist_per_step`` and
``RK_cheat_factor``, the list cadence, the grid (``n_grid``, ``grid_factor``:
the radius of the chain-motor lists) and the walls switch.  Inside a
reference checkout ``updates.install`` points the step at that checkout's
own ``config`` module, which its ``configure`` and ``grid_list_setup`` fill;
without one, a caller sets these names here.
"""
from __future__ import annotations

import numpy as np

dim = 2
Lx = 1.
SRK_order = 2
max_dist_per_step = 1
RK_cheat_factor = 1
n_steps_update_grid_list = 1
grid_factor = 2.
n_grid = 0  # cells per side of the reference's grid (grid_list_setup); motors need it
walls = np.array([False, False, False])
