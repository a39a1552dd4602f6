"""Block-diagonal exchange specs (utils.py:206-311) on the GPU."""


def build_fock_block_specs(P, **kwargs):
    raise NotImplementedError("exchange_block_specs is not implemented on the GPU path yet")
