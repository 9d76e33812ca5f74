"""Placeholder replaced below."""


def build():
    return None
