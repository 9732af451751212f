"""mlem_b200 -- B200-native MLEM reconstruction, a drop-in for the hot path
of the reference's seqcsr4mlem / openmpcsr4mlem.

The compute path is the CUDA library lib/libmlem_b200.so behind the C ABI in
include/mlem_b200.h; `mlem_b200.api` is its Python host layer,
`mlem_b200.synth` builds the synthetic workloads, `mlem_b200.formats` reads
and writes the reference's files, and bin/mlem_b200 is the command-line
drop-in.  Importing the package loads nothing native; the first API call does.
"""
__all__ = ["api", "formats", "synth"]
__version__ = "0.1.0"
