// definitions are in params.h
