"""Helpers for the GPU tests: device copies through torch (plumbing only)."""
import numpy as np
import torch


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def ptr(t):
    return t.data_ptr()


def stream():
    return torch.cuda.current_stream().cuda_stream


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()
