// Stand-in for quill/LogMacros.h (logging is dropped in the parity-pin build).
#pragma once
