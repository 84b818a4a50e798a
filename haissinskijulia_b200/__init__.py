"""B200-native (sm_100a) longitudinal tracking for HaissinskiJulia's
longitudinal_evolve! path, behind a C ABI (include/haissinski_gpu.h).

The compute path is libhaissinski_gpu.so (hand-written CUDA); this package
is the host-side mirror of the reference's Julia API over that library.
"""
from .api import (  # noqa: F401
    ELECTRON_CHARGE,
    MASS_ELECTRON,
    SPEED_LIGHT,
    Batch,
    BinGrid,
    Checkpoint,
    Context,
    EvolveResult,
    HaissinskiError,
    Particles,
    ResidentBunch,
    SimulationBuffers,
    ShardedBunch,
    SimulationParameters,
    WakeModel,
    apply_wakefield_inplace,
    calc_rf_factor,
    calculate_local_histogram,
    create_simulation_buffers,
    gaussian_bunch,
    generate_particles,
    generate_particles_device,
    gaussian_draws,
    longitudinal_evolve,
    next_power_of_two,
    phase_advance,
    quantum_excitation,
    rf_kick,
    synchrotron_radiation,
    synthetic_bunch,
    wake_potential,
    z_to_ϕ,
    ϕ_to_z,
)
from .rings import benchmark_ring, reference_ring  # noqa: F401

__version__ = "0.1.0"
