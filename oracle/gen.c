int x;
