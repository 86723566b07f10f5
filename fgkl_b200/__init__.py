"""fgkl_b200: fgkl's PairHMM / PD-HMM likelihood path on NVIDIA B200 (sm_100a).

The compute path is ``libfgkl_b200.so`` (CUDA kernels + C ABI, ``include/fgkl_b200.h``); this package
is its host-side mirror of fgkl's Rust API (``crates/pairhmm/src/lib.rs``, ``pd.rs``).
"""
from .pairhmm import (  # noqa: F401
    ALT_A, ALT_C, ALT_G, ALT_T, DEL_END, DEL_START, SNP, BatchContext, Config, DeviceError, EmptyHaplotype, EmptyRead,
    MismatchedHaplotypeArrays, MismatchedReadArrays, OutputLength, PairHmm, PairHmmError, PdHaplotype, PdPairHmm, Plan,
    Precision, Read, SharedColumns, plan, shared_columns, NORMAL, INSIDE_DEL, AFTER_DEL, PdPlan, pd_plan, pd_row_states,
    pd_match_accepts, set_call_combining, call_combining_stats, set_allocation_limit,
)
