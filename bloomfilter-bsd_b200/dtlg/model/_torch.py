"""torch, imported on first use (device buffers and streams only)."""


def torch_mod():
    import torch
    return torch
