"""Units (src/Units.jl:7-22)."""
meter = meters = 1.0
kilometer = kilometers = 1000.0
second = seconds = 1.0
minute = minutes = 60.0
hour = hours = 60 * minute
day = days = 24 * hour
KiB = 1024
MiB = 1024 ** 2
GiB = 1024 ** 3
TiB = 1024 ** 4
