"""CPU restatement of the schedule network -- TEST INFRASTRUCTURE ONLY.

The network of graph-intermedia-representation_b200/csrc/sched.cu in float64 numpy: 8 features
-> 32 tanh units -> 12 logits, parameters laid out W1[32][8], b1[32], W2[12][32], b2[12]; loss =
mean softmax cross-entropy. The GPU tests check the device forward pass and gradient against it.
(The schedule network has no counterpart in the reference, which uses fixed thresholds.)
"""
import numpy as np

IN, HID, OUT = 8, 32, 12
NP = HID * IN + HID + OUT * HID + OUT


def unpack(p):
    p = np.asarray(p, np.float64)
    W1 = p[:HID * IN].reshape(HID, IN)
    b1 = p[HID * IN:HID * IN + HID]
    W2 = p[HID * IN + HID:HID * IN + HID + OUT * HID].reshape(OUT, HID)
    b2 = p[HID * IN + HID + OUT * HID:]
    return W1, b1, W2, b2


def forward(p, x):
    W1, b1, W2, b2 = unpack(p)
    h = np.tanh(np.asarray(x, np.float64) @ W1.T + b1)
    return h @ W2.T + b2, h


def loss_and_grad(p, x, y):
    x = np.asarray(x, np.float64)
    y = np.asarray(y)
    n = len(x)
    W1, b1, W2, b2 = unpack(p)
    z, h = forward(p, x)
    z = z - z.max(1, keepdims=True)
    e = np.exp(z)
    sm = e / e.sum(1, keepdims=True)
    loss = float(-np.log(sm[np.arange(n), y]).mean())
    d = sm.copy()
    d[np.arange(n), y] -= 1.0
    d /= n
    gW2 = d.T @ h
    gb2 = d.sum(0)
    dz = (d @ W2) * (1 - h * h)
    gW1 = dz.T @ x
    gb1 = dz.sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2])
