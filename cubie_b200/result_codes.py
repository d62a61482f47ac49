"""Per-run status bits, identical in value to the reference's
``CUBIE_RESULT_CODES`` (``src/cubie/result_codes.py:21-61``)."""

from enum import IntFlag


class CUBIE_RESULT_CODES(IntFlag):
    SUCCESS = 0
    MAX_NEWTON_ITERATIONS_EXCEEDED = 2
    MAX_LINEAR_ITERATIONS_EXCEEDED = 4
    STEP_TOO_SMALL = 8
    DT_EFF_EFFECTIVELY_ZERO = 16
    MAX_LOOP_ITERS_EXCEEDED = 32
    STAGNATION = 64
    BICGSTAB_BREAKDOWN = 128
    NEWTON_DIVERGENCE = 256


def decode_status_codes(status_codes):
    """Map run index -> names of the status bits set (successful runs omitted)."""
    messages = {}
    if status_codes is None:
        return messages
    flags = [f for f in CUBIE_RESULT_CODES if f.value != 0]
    for run_index, code in enumerate(status_codes):
        code = int(code)
        if code == 0:
            continue
        messages[run_index] = [f.name for f in flags if code & f.value == f.value]
    return messages


__all__ = ["CUBIE_RESULT_CODES", "decode_status_codes"]
