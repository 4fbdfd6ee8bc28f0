"""Tamaki PACE-2017 ordering needs a Java solver that is not in this image."""


def get_upper_bound_peo_pace2017(graph, method='tamaki', wait_time=5):
    raise NotImplementedError('the Tamaki ordering needs the Java PACE-2017 solver')
