"""Train the warm-start network on LBM steady states and evaluate it (run on a B200).

    python -m water_flow_simulation_b200.train_warmstart --train 256 --test 32 --epochs 20 \
        --out water_flow_simulation_b200/data/warmstart_net.npz --report report.json

Training cases are seeds 10000.., held-out cases seeds 20000.. (water_flow_simulation_b200.
warmstart.random_case); the report holds the loss history, the held-out loss with and
without training, and the evaluation of the chosen method against the reference protocol.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=256)
    ap.add_argument("--test", type=int, default=32)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--tol", type=float, default=5e-3, help="convergence: window-mean discharge change")
    ap.add_argument("--eval-cases", type=int, default=16)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "data", "warmstart_net.npz"))
    ap.add_argument("--report", default=None)
    args = ap.parse_args()

    import torch
    from . import warmstart as ws
    from .surrogate import SurrogateNet

    log = lambda s: print(f"[{time.strftime('%H:%M:%S')}] {s}", flush=True)  # noqa: E731
    t0 = time.time()
    train = ws.generate(list(range(10000, 10000 + args.train)), log=log)
    test = ws.generate(list(range(20000, 20000 + args.test)), log=log)
    t_gen = time.time() - t0
    net = SurrogateNet(seed=0)
    log(f"network: {net.n_params} parameters")

    def held_out_loss():
        losses = []
        for f, d, t, m in test:
            out = net.forward(torch.as_tensor(f, device=net.device), d)
            p = out[:, :4].cpu().numpy() * net.out_scale[None, :]
            w = m[:, None]
            losses.append(float((w * (p - t) ** 2).sum() / max(w.sum(), 1)))
        return float(np.mean(losses))

    def zero_loss():
        return float(np.mean([float((m[:, None] * t ** 2).sum() / max(m.sum(), 1)) for _, _, t, m in test]))

    net.out_scale = ws.target_scale(train)
    untrained = held_out_loss()
    t1 = time.time()
    hist = ws.train(net, train, epochs=args.epochs, lr=args.lr, log=log)
    torch.cuda.synchronize()
    t_train = time.time() - t1
    trained = held_out_loss()
    log(f"held-out loss: zero prediction {zero_loss():.4f}, untrained {untrained:.4f}, trained {trained:.4f}")
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    st = net.state()
    arrays = {f"{k}_{p}": v[p].numpy().astype(np.float32) for k, v in st.items() for p in ("W", "b")}
    np.savez_compressed(args.out, out_scale=net.out_scale, **arrays)
    ev = ws.evaluate(net, list(range(30000, 30000 + args.eval_cases)), tol=args.tol, log=log)
    report = dict(train_cases=args.train, test_cases=args.test, epochs=args.epochs, params=net.n_params,
                  generate_seconds=t_gen, train_seconds=t_train, loss_history=hist,
                  held_out_loss=dict(zero_prediction=zero_loss(), untrained=untrained, trained=trained),
                  evaluation=ev)
    if args.report:
        with open(args.report, "w") as fh:
            json.dump(report, fh, indent=1)
    log(json.dumps({k: v for k, v in report.items() if k != "loss_history"})[:2000])


if __name__ == "__main__":
    main()
