// Empty stand-in: included by the reference's C0Expansion headers, nothing used.
#pragma once
