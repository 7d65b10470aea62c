"""Drop-in for the reference's ``tr_csr_fp16`` package (spmm/tr_csr_fp16/):
dataset loading, routing and the routed forward driver, on libtrspmm."""
