"""forcepho_b200: forcepho's proposal-evaluation hot path on B200 (sm_100a).

Given a packed patch and a proposal of Sersic source parameters, compute chi2
and d chi2 / d theta per band with hand-written CUDA kernels, behind the
reference's ``Proposer.evaluate_proposal`` / ``Patch`` / ``Posterior`` surface.
"""

__version__ = "0.1.0"

from . import kernel_limits  # noqa: F401
from .proposal import (GPUProposer, Proposer, ProposerBase,  # noqa: F401
                       response_struct_dtype, source_struct_dtype)
