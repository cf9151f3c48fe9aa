"""pacuda-b200: a B200-native recurrence runner, a drop-in for pacuda's librecurrence.so."""
