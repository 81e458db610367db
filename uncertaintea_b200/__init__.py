"""B200-native (sm_100a) batched density + sampler hot path of UncertainTea.

Public surface mirrors the reference's ``UncertainTea.Device`` and
``UncertainTea.Inference`` facades (src/UncertainTea.jl:101-200) for the
device path: batched logjoint / gradient, batched HMC, persistent NUTS,
ChEES-HMC, MEADS, mean-field ADVI, the Philox4x32-10 stream and the R-hat / ESS
diagnostics; plus
the learned gradient surrogate for ChEES-HMC and many-model batched NUTS
(no reference counterparts).
"""
from .models import (BernoulliBeta, BernoulliLogitGLM, HierarchicalNormalNoncentered, LognormalGammaNormal,
                     NormalKnownScale, NormalLocationScale, StudentTHeavyTail, TeaModelSpec, gauss_data, hierarchical_data, logistic_regression_data)
from .device import (DeviceBatchedWorkspace, device_batched_logjoint, device_batched_logjoint_,
                     device_batched_logjoint_gradient, device_batched_logjoint_gradient_, device_lowering_report)
from .inference import HMCChains, batched_chees, batched_hmc, batched_nuts, posterior_array
from .diagnostics import SamplerWarnings, check_diagnostics, ess, has_warnings, min_ess_per_second, rhat, summarize
from .surrogate import GradientSurrogate, batched_chees_surrogate
from .multi import MultiChains, MultiModelBatch, batched_nuts_multi
from .vi import ADVIResult, batched_advi, variational_mean, variational_samples
from .meads import batched_meads
from . import rng

__all__ = [
    "BernoulliBeta", "BernoulliLogitGLM", "HierarchicalNormalNoncentered", "LognormalGammaNormal",
    "NormalKnownScale", "NormalLocationScale", "StudentTHeavyTail", "TeaModelSpec",
    "gauss_data",
    "hierarchical_data",
    "logistic_regression_data", "DeviceBatchedWorkspace", "device_batched_logjoint", "device_batched_logjoint_",
    "device_batched_logjoint_gradient", "device_batched_logjoint_gradient_", "device_lowering_report", "HMCChains",
    "batched_chees", "batched_hmc", "batched_nuts", "posterior_array", "ess", "min_ess_per_second", "rhat",
    "summarize", "check_diagnostics", "has_warnings", "SamplerWarnings", "rng", "GradientSurrogate", "batched_chees_surrogate", "MultiChains", "MultiModelBatch",
    "batched_nuts_multi", "ADVIResult", "batched_advi", "variational_mean", "variational_samples",
    "batched_meads",
]
