"""Host-resident batches: simulate images whose parameters and outputs live in
pinned host memory, overlapping host->device copies, the slice + CTF
launches and device->host copies on two CUDA streams.

This is the end-to-end form of a batched ``simulate`` call when the caller
holds its poses and CTF parameters on the host and wants the image stack
back on the host.
"""

from __future__ import annotations

import numpy as np

from . import _native as nat


class HostStreamingSimulator:
    """Two-stream pipeline over sub-batches of ``sub_batch`` images."""

    def __init__(self, volume, image_config, integrator, flags, *, sub_batch=2048, images_per_chunk=0,
                 sort_orientations=True):
        import torch

        self.torch = torch
        self.volume = volume
        self.cfg = image_config
        self.integrator = integrator
        self.flags = flags
        self.sub_batch = int(sub_batch)
        self.chunk = images_per_chunk
        self.sort = sort_orientations
        self.order_d = [None, None]
        dev = volume.device
        py, px = image_config.padded_shape
        self.out_shape = (py, px // 2 + 1)
        self.streams = [torch.cuda.Stream(device=dev) for _ in range(2)]
        self.params_d = [torch.empty((self.sub_batch, nat.PARAMS_DOUBLES), dtype=torch.float64, device=dev)
                         for _ in range(2)]
        self.out_d = [torch.empty((self.sub_batch,) + self.out_shape, dtype=torch.complex64, device=dev)
                      for _ in range(2)]
        desc = nat.make_desc(volume.shape[0], py, px, flags, integrator.fill_value, images_per_chunk)
        ws = nat.workspace_size(desc, self.sub_batch)
        self.ws = [torch.empty(max(ws, 1), dtype=torch.uint8, device=dev) for _ in range(2)]

    @staticmethod
    def pinned_params(params: np.ndarray):
        import torch

        t = torch.empty(params.shape, dtype=torch.float64, pin_memory=True)
        t.copy_(torch.from_numpy(np.ascontiguousarray(params)))
        return t

    def pinned_output(self, n):
        return self.torch.empty((n,) + self.out_shape, dtype=self.torch.complex64, pin_memory=True)

    def sub_batches(self, n):
        """(start, count) of each sub-batch: sub_batch / 8, / 4, / 2, then full ones.

        Every call is ordered after the caller's stream, so its first
        device-to-host copy waits for its first sub-batch's simulation; the
        ramp keeps that wait to a small batch's instead of a full one's.
        """
        out, pos, size = [], 0, max(1, self.sub_batch // 8)
        while pos < n:
            cnt = min(size, n - pos)
            out.append((pos, cnt))
            pos += cnt
            size = min(self.sub_batch, 2 * size)
        return out

    def run(self, params_host, out_host):
        """params_host: pinned float64 [n, 32]; out_host: pinned complex64 [n, Py, Px//2+1].

        With ``sort_orientations`` each sub-batch is processed in
        orientation order (outputs still land in their own slots).
        """
        torch = self.torch
        n = params_host.shape[0]
        batches = self.sub_batches(n)
        orders = []
        if self.sort:
            from .simulator import orientation_order

            rots = params_host[:, 0:9].numpy().reshape(-1, 3, 3)
            for s0, cnt in batches:
                o = orientation_order(rots[s0:s0 + cnt])
                orders.append(torch.from_numpy(o).pin_memory())
        cur = torch.cuda.current_stream()
        for s in self.streams:
            s.wait_stream(cur)
        for i, (s0, cnt) in enumerate(batches):
            k = i % 2
            st = self.streams[k]
            with torch.cuda.stream(st):
                pd = self.params_d[k][:cnt]
                od = self.out_d[k][:cnt]
                pd.copy_(params_host[s0:s0 + cnt], non_blocking=True)
                od_order = None
                if self.sort:
                    if self.order_d[k] is None:
                        self.order_d[k] = torch.empty(self.sub_batch, dtype=torch.int32, device=pd.device)
                    od_order = self.order_d[k][:cnt]
                    od_order.copy_(orders[i], non_blocking=True)
                self.integrator.run(self.volume, self.cfg, None, self.flags, params_device=pd, out=od,
                                    workspace=self.ws[k], stream=st, images_per_chunk=self.chunk, n=cnt,
                                    order=od_order)
                out_host[s0:s0 + cnt].copy_(od, non_blocking=True)
        for s in self.streams:
            cur.wait_stream(s)
        return out_host
