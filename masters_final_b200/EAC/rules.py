"""k-range rules for the ensemble (MyML/MyML/EAC/rules.py:17-53)."""
import numpy as np


def rule1(n):
    """sqrt: [ceil(sqrt(n)/2), ceil(sqrt(n))]"""
    return [int(np.ceil(v)) for v in (np.sqrt(n) / 2, np.sqrt(n))]


def rule2(n):
    """2sqrt"""
    return [x * 2 for x in rule1(n)]


def rule3(n, sk, th):
    """fixed s/k"""
    return [int(np.ceil(v)) for v in (n * 1.0 / sk, th * n * 1.0 / sk)]


def sk1(n):
    """sqrt/2"""
    return int(np.sqrt(n) / 2)


def rule4(n):
    """sk=sqrt_2, th=30%"""
    return rule3(n, sk1(n), 1.3)


def rule5(n):
    """sk=300, th=30%"""
    return rule3(n, 300, 1.3)


def rule6(n, th=1.3):
    """sqrt * log10, th=30%"""
    kmin = np.sqrt(n) * np.log10(n) / 2
    return [int(kmin), int(kmin * th)]
