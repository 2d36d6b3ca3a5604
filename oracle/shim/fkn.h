/* Empty stand-in for the FKN application header (MFC app class, not needed by spars.cpp). */
#pragma once
