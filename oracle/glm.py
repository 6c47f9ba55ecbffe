"""TEST INFRASTRUCTURE — dense CPU restatement of the reference's GLM fits (numpy).

Only tests/ and bench.py's CPU legs use this module, as the checker; the product (fereg_b200)
never imports it.

The Poisson and logit MLEs with absorbed fixed effects are unique, so the dense restatement fits
the same model with explicit FE dummies: IRLS on the full design (glm/irls.rs:367-560 with the
families of glm/family.rs:101-147: Poisson w = mu, z = eta - 1 + y / mu; logit w = mu (1 - mu),
z = eta + (y - mu) / w) until the deviance stops changing (relative 1e-15). The variance follows
glm/mod.rs:1-22: X~ is X residualized on the dummies with the final weights, robust
(X~'WX~)^-1 [sum (y - mu)^2 x~ x~'] (X~'WX~)^-1 N / (N - 1), clustered with G / (G - 1), logit
`oim` the inverse Hessian (X~'WX~)^-1.
"""

import numpy as np
from scipy.special import expit, gammaln


def dense_glm(family, terms, y, X, vce="robust", cl=None, maxiter=200):
    """terms: list of (codes, levels); cl: (codes, G) for vce="cluster". Returns b, V, deviance,
    log-likelihood."""
    n = len(y)
    D = np.concatenate([np.eye(g)[c] for c, g in terms], axis=1)
    Z = np.concatenate([X, D], axis=1)
    if family == "poisson":
        mu = (y + y.mean()) / 2
        eta = np.log(mu)
    else:
        mu = (y + 0.5) / 2
        eta = np.log(mu / (1 - mu))
    dev_old = np.inf
    for _ in range(maxiter):
        if family == "poisson":
            w = mu
            z = eta - 1 + y / mu
        else:
            w = mu * (1 - mu)
            z = eta + (y - mu) / w
        sw = np.sqrt(w)[:, None]
        coef, *_ = np.linalg.lstsq(Z * sw, z * sw[:, 0], rcond=None)
        eta = Z @ coef
        if family == "poisson":
            mu = np.exp(eta)
            dev = 2 * np.sum(np.where(y > 0, y * np.log(np.where(y > 0, y, 1) / mu), 0) - (y - mu))
        else:
            mu = expit(eta)
            dev = -2 * np.sum(y * eta - np.logaddexp(0, eta))
        if abs(dev - dev_old) <= 1e-15 * dev:
            break
        dev_old = dev
    k = X.shape[1]
    b = coef[:k]
    w = mu if family == "poisson" else mu * (1 - mu)
    sw = np.sqrt(w)[:, None]
    cd, *_ = np.linalg.lstsq(D * sw, X * sw, rcond=None)
    Xt = X - D @ cd
    A = np.linalg.inv(Xt.T @ (w[:, None] * Xt))
    s = (y - mu)[:, None] * Xt
    if vce == "oim":
        V = A
    elif vce == "robust":
        V = A @ (s.T @ s) @ A * n / (n - 1)
    else:
        codes, G = cl
        S = np.zeros((G, k))
        np.add.at(S, codes, s)
        V = A @ (S.T @ S) @ A * G / (G - 1)
    if family == "poisson":
        ll = np.sum(y * eta - mu - gammaln(y + 1))
    else:
        ll = np.sum(y * eta - np.logaddexp(0, eta))
    return b, V, dev, ll
