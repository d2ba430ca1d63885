/* join oracle: filled in below */
