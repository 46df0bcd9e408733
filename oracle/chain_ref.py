"""The deform-and-render step through the reference's own kernels (test and
benchmark oracle, never part of the product).

Same composition as ``deepcharacters_b200.chain.DeformRenderChain``: node
skinning on the host (Pose2EmbeddedGraphCpu is a CPU op in the reference,
Pose2EmbeddedGraphCPUOp.cpp:129-300; restated in ``skinning_oracle.pose2eg``),
then the reference CUDA kernels compiled from the reference tree into
oracle/_ref (EmbeddedGraphGPUOp, CUDABasedRasterization, CameraProjectionGPUOp,
Skeletool ProjectedMeshBoundary raster, MultiViewSilhouetteLossGPUOp and their
gradient kernels), driven op by op like the TF graph, with the losses and the
AddN of the two vertex gradients as torch elementwise ops.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O
from . import skinning_oracle as K


class RefChain:
    def __init__(self, sc, dev, frames, views, width, height, w_sil=1e-3, w_sil1=1e-3):
        import torch
        from deepcharacters_b200.chain import character, eg_data
        self.sc, self.dev = sc, dev
        self.B, self.C, self.W, self.H, self.N = frames, views, width, height, int(sc["verts"].shape[0])
        self.w_sil, self.w_sil1 = w_sil, w_sil1
        self.ch = character(sc)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        self.t = t
        self.inp = {k: t(sc[k]) for k in ("dT", "dA", "disp", "colors", "texture", "sh", "extr", "intr", "target",
                                          "dt", "crops")}
        self.r = O.RefRenderer(sc["faces"], sc["texcoords"], self.N, views, width, height, "vertexColor", "shadeless",
                               "none", 2, 2)
        self.eg = O.RefEG(eg_data(sc), dev)
        self.s = O.RefSilhouette()
        self.gm = torch.zeros((frames, len(sc["markers"]), 3), device=dev)

    def step(self, sT=None, sA=None, verts=None, normals=None, raster=None):
        """One step.  ``sT`` / ``sA`` (device [B,M,3]) replace the host node
        skinning when given, ``verts`` / ``normals`` [B,N,3] the deformed mesh
        that the raster and the silhouette see, so that each stage can be
        compared on the device chain's own inputs; ``raster`` (dict with
        bary / face / render / vnormal) replaces the reference raster's outputs
        downstream of it (the loss and the adjoints)."""
        import torch
        sc, i, t = self.sc, self.inp, self.t
        B = self.B
        if sT is None or sA is None:
            hT, hA, _ = K.pose2eg(self.ch, sc["dofs"], sc["graph"].node_vertex, sc["skin_weights"])
            sT, sA = t(hT.astype(np.float32)), t(hA.astype(np.float32))
        eg = self.eg.forward(i["dT"], i["dA"], sT, sA, i["disp"])
        v = eg["vertices"] if verts is None else verts
        nrm = eg["normals"] if normals is None else normals
        fw = self.r.forward(B, v, i["colors"], i["texture"], i["sh"], i["extr"], i["intr"], depth=False, sync_each=0)
        face_ref = fw["face"]
        if raster is not None:
            fw = dict(fw, **raster)
        diff = 255.0 * (fw["render"] - i["target"]) * (fw["face"] >= 0).unsqueeze(-1)
        cnt = torch.count_nonzero(diff).clamp_min(1)
        l1 = diff.abs().sum() / cnt
        g = 255.0 * torch.sign(diff) / cnt
        p2d = self.s.project(v, None, i["extr"], i["intr"], 1)
        n2d = self.s.project(v, nrm, i["extr"], i["intr"], 0)
        isb = O.ref_mesh_boundary(sc["faces"], v, i["extr"], i["intr"], self.W, self.H)
        res, res1, dtg, cid = self.s.forward(p2d, n2d, isb, i["dt"], i["crops"])
        gp = self.s.backward(2 * self.w_sil * res, 2 * self.w_sil1 * res1, dtg, cid, i["crops"])
        gv_sil = self.s.project_grad(gp, v, i["extr"], i["intr"], 1)
        bw = self.r.backward(B, g.contiguous(), v, i["colors"], i["texture"], i["sh"], i["target"], fw["vnormal"],
                             fw["bary"], fw["face"], i["extr"], i["intr"])
        eb = self.eg.backward(bw["vertex_pos_grad"] + gv_sil, self.gm, eg["da"], eg["sa"])
        loss = torch.stack([l1, self.w_sil * (res.double() ** 2).sum().float(),
                            self.w_sil1 * (res1.double() ** 2).sum().float()])
        return dict(sT=sT, sA=sA, v=eg["vertices"], n=eg["normals"], face=face_ref, bary=fw["bary"], render=fw["render"],
                    p2d=p2d, isb=isb, res=res, res1=res1, cid=cid, gv_sil=gv_sil, gv=bw["vertex_pos_grad"] + gv_sil,
                    gcol=bw["vertex_color_grad"], gT=eb["t"], gA=eb["r"], loss=loss)
