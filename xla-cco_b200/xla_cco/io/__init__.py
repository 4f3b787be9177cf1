"""File formats: ConfigPack (configurations) and C++-style function tables."""

from xla_cco.io.configpack import (
    PackedConfig,
    read_configpack,
    stack_fractional,
    write_configpack,
)
from xla_cco.io.tables import write_function_table

__all__ = ["PackedConfig", "read_configpack", "stack_fractional", "write_configpack",
           "write_function_table"]  # fmt: skip
