"""B200-native static structure factor S(q) for sqcalc: the NUFFT hot path of
``sqcalc static`` as hand-written sm_100a CUDA behind a C ABI (libsqnufft.so)."""
