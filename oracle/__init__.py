"""The oracle: CPU restatements of AR_Sim's per-step path used to check the CUDA library.

TEST INFRASTRUCTURE ONLY.  ``oracle.cpu`` wraps this repository's C restatement
(``oracle.c``); ``oracle.ref`` wraps the reference's own kernel bodies compiled for the CPU
(``ref_build.py`` -> ``_ref/libref_cpu.so``), which pins the restatement.  Only tests/,
bench.py's CPU legs and __graft_entry__.smoke() import this package.
"""
