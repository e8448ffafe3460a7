/* Empty stand-in for an absent third-party header (oracle build only). */
#pragma once
