"""B200-native stepper of the gtdgl (juliaTDGL 2) ladder cycle.

Host side: the model, grid, masks and Stepper set-up of the reference (``model``, ``grid``, ``scheme``,
``state``).  Device side: the CUDA library ``libtdgl_b200.so`` behind the C-ABI of ``include/tdgl_b200.h``,
driven from Python through ``gpu`` (the accelerator interface of the reference's TDGLGPU module).
"""
from .model import Band, Model, two_band, equilibrium, eps_band, stiffness
from .grid import Grid, Masks, GeomSpec, box_masks, build_masks, slab_thickness
from .state import State, initial_state
from .scheme import Stepper, selffield, RKCCoef, Heat, QPExchange, QPExchangeN
