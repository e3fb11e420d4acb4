def enable():
    return None


def disable():
    return None
