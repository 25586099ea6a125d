/* POSIX stand-in (empty) for the ATL conversion header (oracle test infrastructure only). */
#pragma once
