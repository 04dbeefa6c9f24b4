"""Level-set (embedded) wake: the sheet's level set, the cut-element census
with the extended DOFs, and the multivalued operator over the device
Picard and upwind operators (pyfp3d/wake/)."""

from .cut_elements import CutElementMap
from .levelset import WakeLevelSet
from .multivalued import MultivaluedOperator

__all__ = ["CutElementMap", "MultivaluedOperator", "WakeLevelSet"]
