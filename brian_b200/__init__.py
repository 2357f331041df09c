"""brian_b200 -- Brian 1's clock-driven simulation loop on NVIDIA B200.

Drop-in for the reference's NeuronGroup / Connection / DelayConnection /
ExponentialSTDP / Network.run / SpikeMonitor / StateMonitor / modelfitting
path: ``from brian_b200 import *`` gives the same names; the simulation runs
in hand-written sm_100a kernels behind the C ABI of include/brian_b200.h.
"""
from numpy import *  # noqa: F401,F403  (the reference re-exports numpy)
from numpy.random import rand, randn, seed  # noqa: F401
from .units import *  # noqa: F401,F403
from . import units
from .clock import Clock, defaultclock, reinit_default_clock, guess_clock, define_default_clock
from .equations import Equations
from .groups import (NeuronGroup, PoissonGroup, SpikeGeneratorGroup, Threshold, VariableThreshold,
                     PoissonThreshold, NoThreshold, StringThreshold, Reset, VariableReset, StringReset, NoReset,
                     Refractoriness, LazyStateUpdater, EmpiricalThreshold)
from .connections import Connection, DelayConnection, IdentityConnection
from .stdp import ExponentialSTDP, STDP
from .synapses import Synapses
from .monitors import (SpikeMonitor, StateMonitor, RecentStateMonitor, ISIHistogramMonitor, SpikeCounter,
                       PopulationSpikeCounter,
                       PopulationRateMonitor,
                       CoincidenceCounter, MultiStateMonitor)
from .network import (Network, MagicNetwork, run, reinit, stop, clear, network_operation, NetworkOperation,
                      set_global_preferences, get_global_preference)
from .batch import NetworkBatch
from .timedarray import TimedArray, TimedArraySetter, set_group_var_by_array
from .statistics import firing_rate, CV, gamma_factor, get_gamma_factor, spike_triggered_average
from .modelfitting import (GPUModelFitting, modelfitting, distributed_modelfitting, get_spikes, predict, print_table, PSO, GA, CMAES,
                           OptimizationResult, euler_scheme, rk2_scheme, exp_euler_scheme)

__version__ = "0.1.0"
