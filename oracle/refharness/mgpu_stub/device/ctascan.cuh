// Empty stand-in: the reference includes moderngpu (mergekernel.cuh:13-16) but calls none of it.
