"""Generates tests/golden/loss_pyramid.pt from the reference's own loss
module (pyTensorRay/loss.py, which needs only torch): seeded images and
targets of an odd and an even size, the L1/L2 losses and their pyramid
forms, and each loss's image gradient. Run in a checkout where the
reference sits at /root/reference:

    python tests/golden/make_loss_goldens.py
"""
import importlib.util
import os

import torch

REF = "/root/reference/pyTensorRay/loss.py"
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "loss_pyramid.pt")


def main():
    spec = importlib.util.spec_from_file_location("ref_loss", REF)
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    g = torch.Generator().manual_seed(11)
    cases = []
    for h, w in [(37, 23), (32, 20), (5, 9)]:
        img = torch.rand(h, w, 3, generator=g)
        tgt = torch.rand(h, w, 3, generator=g)
        img[h // 2, w // 3, 1] = float("nan")
        weight = 0.75
        case = {"img": img.clone(), "target": tgt.clone(), "weight": weight}
        tp = ref.build_pyramid(tgt)
        case["levels"] = len(tp)
        for name, fn, t in [("l1", ref.compute_render_loss_L1, tgt), ("l2", ref.compute_render_loss_L2, tgt),
                            ("pyramid_l1", ref.compute_render_loss_pyramid_L1, tp),
                            ("pyramid_l2", ref.compute_render_loss_pyramid_L2, tp)]:
            x = img.clone().requires_grad_(True)
            loss = fn(x, t, weight)
            loss.backward()
            case[name] = (float(loss.detach()), x.grad.clone())
        cases.append(case)
    torch.save(cases, OUT)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
