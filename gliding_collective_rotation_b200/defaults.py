"""Option defaults of the step path, with the GPU switches.

``set_defaults()`` returns ``(sim, help)`` like the reference's
``defaults.set_defaults`` (defaults.py:12-255): the keys the step path and
its set-up read, with the reference's names, defaults and value types
(the type of each default is the command-line type), plus

* ``gpu``            run ``updates.SRK2_force_calc`` on the B200 path;
* ``gpu_precision``  ``'fp64'`` or ``'mixed'`` (FP32 forces, FP64 positions);
* ``gpu_noise``      ``'philox'`` (counter-based stream on the device) or
                     ``'mt'`` (the reference's MT19937 stream seeded with
                     ``seed``, drawn on the host and injected);
* ``gpu_cell_factor`` GPU cell side as a multiple of the pair cutoff (>= 1);
* ``gpu_steps_per_graph`` steps per captured CUDA graph.
"""
import numpy as np


def set_defaults():
    sim, help = {}, {}
    sim['filelabel'] = 'most_recent'
    help['filelabel'] = 'Label that names the files of a run.'
    sim['n_threads'] = 3
    help['n_threads'] = 'Number of threads used to calculate forces (CPU path).'
    sim['dim'] = 2
    help['dim'] = 'Number of spatial dimensions: 2 or 3.'
    sim['SRK_order'] = 2
    help['SRK_order'] = 'Stochastic Runge-Kutta order of the step: 2 or 4.'
    sim['Lx'] = 50.
    help['Lx'] = 'Side of the periodic box (the same along every axis).'
    sim['walls'] = 'none'
    help['walls'] = 'Boundary conditions (the GPU path is periodic only).'
    sim['bead_density'] = 0.5
    help['bead_density'] = 'Initial placement: beads per unit area.'
    sim['chain_length'] = 10
    help['chain_length'] = 'Beads per chain.'
    sim['n_chains'] = -1
    help['n_chains'] = 'Initialization: Number of chains. If positive, overrides bead_density.'
    sim['t_max'] = -1
    help['t_max'] = 'Stopping conditions: maximum time. Negative for infinity.'
    sim['stepnum_max'] = -1
    help['stepnum_max'] = 'Stopping conditions: maximum step number. Negative for infinity.'
    sim['dtmax'] = 4.e-3
    help['dtmax'] = 'Upper bound of the adaptive time step (RK_cheat_factor multiplies it afterwards).'
    sim['dt0'] = 0.0001 * sim['dtmax']
    help['dt0'] = 'Small timestep to use in first update only.'
    sim['RK_cheat_factor'] = 1.
    help['RK_cheat_factor'] = 'Take a step this many times larger than the test step used for forces.'
    sim['timestep_safety_factor'] = 0.025
    help['timestep_safety_factor'] = 'Adaptive timestep: fraction of the smallest length allowed per update.'
    sim['n_grid_max'] = 0
    help['n_grid_max'] = 'Maximum number of grid cells per side (0: no limit).'
    sim['n_grid_min'] = 1
    help['n_grid_min'] = 'Minimum number of grid cells per side.'
    sim['grid_factor'] = 2.
    help['grid_factor'] = 'Safety factor for deciding grid spacing.'
    sim['T'] = 1e-3
    help['T'] = "Boltzmann's constant times temperature, k_B T"
    sim['repel_d_max'] = 1.
    help['repel_d_max'] = 'WCA: steric repulsion diameter of beads.'
    sim['WCA_epsilon'] = 1.
    help['WCA_epsilon'] = 'WCA: strength of potential.'
    sim['WCA_shift'] = 0.0 * sim['repel_d_max']
    help['WCA_shift'] = 'WCA: shift of dependence on distance.'
    sim['LJ_cutoff_factor'] = 1.
    help['LJ_cutoff_factor'] = 'WCA: cutoff distance (1: purely repulsive; >= 2: LJ attraction).'
    sim['n_nearby_beads_dont_repel'] = 4
    help['n_nearby_beads_dont_repel'] = 'WCA off between beads this close on the same chain (<0: whole chain).'
    sim['b_FENE'] = False
    help['b_FENE'] = 'Linear springs: FENE instead of Hookean (not on the GPU path).'
    sim['k'] = 100.
    help['k'] = 'Linear springs: spring constant.'
    sim['a'] = 0.5
    help['a'] = 'Linear springs: rest length.'
    sim['kappa'] = 1e1
    help['kappa'] = 'Stiffness of the bending springs (negative: rigid rods).'
    sim['spontaneous_bond_angle'] = 0.0 * np.pi
    help['spontaneous_bond_angle'] = 'Bending springs: offset angle to zero of potential.'
    sim['rigid_rod_projection_factor'] = 0.
    help['rigid_rod_projection_factor'] = 'Weight of the rigid-rod motion blended into each chain update (1: rigid rods).'
    sim['FENE_tolerance'] = 0.1
    help['FENE_tolerance'] = 'FENE maximum extension (not on the GPU path).'
    sim['v0'] = 1.
    help['v0'] = 'Self-propulsion: force.'
    sim['v_tan_angle'] = 0.0 * np.pi
    help['v_tan_angle'] = 'Self-propulsion: angle offset of active force relative to tangent.'
    sim['b_use_tangent_as_propulsion_direction'] = True
    help['b_use_tangent_as_propulsion_direction'] = 'Propel along the tangent (True) or a diffusing direction.'
    sim['sliding_partner_maxdist'] = 0.
    help['sliding_partner_maxdist'] = 'Active sliding partner distance (not on the GPU path).'
    sim['t_wait_v0'] = -1.
    help['t_wait_v0'] = 'Early times: wait until this time before turning on self-propulsion.'
    sim['seed'] = 0
    help['seed'] = 'Noise: seed for random number generator for reproducible runs.'
    sim['D'] = -1.
    help['D'] = 'Noise: translational diffusion constant; negative: kT/r.'
    sim['Dr'] = -1.
    help['Dr'] = 'Noise: rotational diffusion constant; negative: 3 D / (4 r^2).'
    sim['pos_init_noise'] = 1.
    help['pos_init_noise'] = 'Initialization: translational noise about the box centre, scaled by size.'
    sim['phi_init'] = 0.
    help['phi_init'] = 'Initialization: reference initial angle for all chains.'
    sim['phi_init_noise'] = 1.e5
    help['phi_init_noise'] = 'Initialization: angular noise of initial chain angles.'
    sim['a_init_factor'] = 1.e-8
    help['a_init_factor'] = 'Initialization: shrink chain rest lengths by this fraction before growing.'
    sim['t_init_grow'] = 1.
    help['t_init_grow'] = 'Initialization: time for chains to grow to their regular length.'
    sim['b_grow'] = False
    help['b_grow'] = 'Growth and division of chains (not on the GPU path).'
    sim['n_motors'] = 0
    help['n_motors'] = 'Motors: total number (not on the GPU path).'
    sim['motor_density'] = 0.
    help['motor_density'] = 'Motors: area density (not on the GPU path).'
    sim['ticker_every'] = 1000
    help['ticker_every'] = 'Interval in steps for printing status info.'
    sim['resultspath'] = './Results/'
    help['resultspath'] = 'Folder the run writes its files to.'
    sim['save_state_every'] = -1.
    help['save_state_every'] = 'Time interval between saved states; negative: never.'
    sim['plot_every'] = -1
    help['plot_every'] = 'Plot interval in steps (plots are not part of this package).'
    # GPU switches
    sim['gpu'] = True
    help['gpu'] = 'Run the step on the B200 path.'
    sim['gpu_precision'] = 'fp64'
    help['gpu_precision'] = "'fp64' or 'mixed' (FP32 forces and SRK arithmetic, FP64 positions)."
    sim['gpu_noise'] = 'philox'
    help['gpu_noise'] = "'philox' (device stream) or 'mt' (reference MT19937 stream, host-drawn)."
    sim['gpu_cell_factor'] = 1.0
    help['gpu_cell_factor'] = 'GPU cell side as a multiple of the pair cutoff (>= 1).'
    sim['gpu_steps_per_graph'] = 10
    help['gpu_steps_per_graph'] = 'SRK2 steps per captured CUDA graph.'
    return sim, help
