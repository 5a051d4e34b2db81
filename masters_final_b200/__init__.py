"""masters_final_b200: the evidence accumulation clustering (EAC) hot path of
diogo-aos/masters_final, rebuilt for NVIDIA B200 (sm_100a).

Drop-in modules mirror the reference's import paths:

    masters_final_b200.cluster.KMeans            K_Means
    masters_final_b200.utils.partition           generateEnsemble, convertClusterStringToIndex
    masters_final_b200.utils.scan                scan_gpu, exprefixsumNumba, exprefixsumNumbaSingle
    masters_final_b200.graph.mst                 boruvka_minho_gpu
    masters_final_b200.graph.connected_components connected_comps_gpu
    masters_final_b200.EAC.sparse                EAC_CSR
    masters_final_b200.EAC.eac                   EAC, sp_sl_lifetime, lifetime_n_clusters
    masters_final_b200.EAC.rules                 rule1 ...

All compute runs in libeacb200.so (hand-written CUDA for sm_100a) through the C
ABI in include/eacb200.h; PyTorch tensors serve as device buffers only.
"""
__version__ = "0.1.0"
