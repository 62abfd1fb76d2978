"""Two forward calls of tigre_conv3d_fwd per U-Net layer shape (128^3 16->16, 64^3 64->64): the
workload of profiles/conv3d_unet_layers.txt."""
import ctypes as C
import os
import sys

import torch
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from tigre_b200 import _native as N
L = N.lib()
p = lambda t: C.c_void_p(t.data_ptr())
for n, cin, cout in [(128, 16, 16), (64, 64, 64)]:
    x = torch.randn(n, n, n, cin, device="cuda").to(torch.bfloat16)
    w = (torch.randn(cout, 27 * cin, device="cuda") / 20).to(torch.bfloat16)
    b = torch.zeros(cout, device="cuda")
    y = torch.empty(n, n, n, cout, device="cuda", dtype=torch.bfloat16)
    col = torch.empty(16, dtype=torch.bfloat16, device="cuda")
    for _ in range(2):
        N.check(L.tigre_conv3d_fwd(p(x), p(w), p(b), p(y), None, n, n, n, cin, cout, 1, p(col), None), "fwd")
    torch.cuda.synchronize()
print("ok")
